// Surface data terms (unoriented varifold, current, measure): face geometry, fused energy (self - 2 cross in
// one pass over the concatenated source faces), fused gradient and the deterministic faces->vertices gather.
// Replaces base/surfaceDistances.py:22-573.
#include <vector>

#include "../../include/lddmm_b200.h"
#include "kernel_ops.cuh"
#include "launch_config.cuh"

namespace lddmm {

// Per-face record (FP64): centre, surfel = cross(v2-v1, v3-v1)/2, unit normal, area a = sqrt(|surfel|^2+1e-10)
// (the reference's regularised area, base/surfaceDistances.py:340), weighted area aw = a fw, face weight fw.
struct FaceRec {
  double c[3], s[3], n[3], a, aw, fw;
};

__global__ void face_geometry_kernel(const double* __restrict__ v, const int64_t* __restrict__ faces,
                                     const double* __restrict__ w, int nf, FaceRec* __restrict__ out) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nf) return;
  const int64_t i0 = faces[3 * f], i1 = faces[3 * f + 1], i2 = faces[3 * f + 2];
  double p0[3], p1[3], p2[3];
  for (int c = 0; c < 3; ++c) {
    p0[c] = v[3 * i0 + c];
    p1[c] = v[3 * i1 + c];
    p2[c] = v[3 * i2 + c];
  }
  FaceRec r;
  const double e1[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
  const double e2[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
  r.s[0] = 0.5 * (e1[1] * e2[2] - e1[2] * e2[1]);
  r.s[1] = 0.5 * (e1[2] * e2[0] - e1[0] * e2[2]);
  r.s[2] = 0.5 * (e1[0] * e2[1] - e1[1] * e2[0]);
  for (int c = 0; c < 3; ++c) r.c[c] = (p0[c] + p1[c] + p2[c]) / 3.0;
  r.a = sqrt(r.s[0] * r.s[0] + r.s[1] * r.s[1] + r.s[2] * r.s[2] + 1e-10);
  for (int c = 0; c < 3; ++c) r.n[c] = r.s[c] / r.a;
  r.fw = w ? (w[i0] + w[i1] + w[i2]) / 3.0 : 1.0;
  r.aw = r.a * r.fw;
  out[f] = r;
}

// Sources = faces of surface A (weight factor 1) followed by faces of surface B (weight factor wB).
struct FaceSources {
  const FaceRec* A;
  int mA;
  const FaceRec* B;
  double wB;
};

__device__ __forceinline__ const FaceRec& src_face(const FaceSources& S, int l, double& fac) {
  if (l < S.mA) {
    fac = 1.0;
    return S.A[l];
  }
  fac = S.wB;
  return S.B[l - S.mA];
}

// Source fields: centre' (0-2), aw * factor (3), unit normal (4-6); current: centre', 0, fw * surfel * factor.
template <int KIND>
__device__ __forceinline__ void face_source_fields(const FaceSources& S, const Frame& f, int l, double* o) {
  double fac;
  const FaceRec& r = src_face(S, l, fac);
  o[0] = (r.c[0] - f.o0) * f.s;
  o[1] = (r.c[1] - f.o1) * f.s;
  o[2] = (r.c[2] - f.o2) * f.s;
  if (KIND == LDDMM_DATA_CURRENT) {
    o[3] = 0.0;
    for (int c = 0; c < 3; ++c) o[4 + c] = fac * r.s[c] * r.fw;
  } else {
    o[3] = fac * r.aw;
    for (int c = 0; c < 3; ++c) o[4 + c] = r.n[c];
  }
}

// Target lane-group state: centre' and the unit normal (varifold, measure) or fw * surfel (current).
template <typename V> struct FaceTgt { V y0, y1, y2, n0, n1, n2; };

template <typename V, int KIND>
__device__ __forceinline__ void load_face_target(const FaceRec* T, const Frame& f, int i0, int i1, FaceTgt<V>& t) {
  const FaceRec &r0 = T[i0], &r1 = T[i1];
  t.y0 = VT<V>::pack((r0.c[0] - f.o0) * f.s, (r1.c[0] - f.o0) * f.s);
  t.y1 = VT<V>::pack((r0.c[1] - f.o1) * f.s, (r1.c[1] - f.o1) * f.s);
  t.y2 = VT<V>::pack((r0.c[2] - f.o2) * f.s, (r1.c[2] - f.o2) * f.s);
  if (KIND == LDDMM_DATA_CURRENT) {
    t.n0 = VT<V>::pack(r0.s[0] * r0.fw, r1.s[0] * r1.fw);
    t.n1 = VT<V>::pack(r0.s[1] * r0.fw, r1.s[1] * r1.fw);
    t.n2 = VT<V>::pack(r0.s[2] * r0.fw, r1.s[2] * r1.fw);
  } else {
    t.n0 = VT<V>::pack(r0.n[0], r1.n[0]);
    t.n1 = VT<V>::pack(r0.n[1], r1.n[1]);
    t.n2 = VT<V>::pack(r0.n[2], r1.n[2]);
  }
}

// ---- energies: dots[k] = weight_k * sum_l e_kl payload_kl. Varifold 13 FP32 + 1 SFU per pair. ----
template <int KIND>
struct OpSurfEnergy {
  static constexpr int NS = 7, NA = (KIND == LDDMM_DATA_CURRENT) ? 3 : 1;
  static constexpr bool kCull = true;  // exact culling of far face tiles
  static constexpr bool kCompInRegisters = true;  // measured faster than shared memory for this op
  struct Params {
    const FaceRec* T;
    FaceSources S;
    double* dots;
    Frame f;
  };
  template <typename V> using Tgt = FaceTgt<V>;
  template <typename V>
  static __device__ __forceinline__ void load_target(const Params& P, int i0, int i1, Tgt<V>& t) {
    load_face_target<V, KIND>(P.T, P.f, i0, i1, t);
  }
  static __device__ __forceinline__ void source_fields(const Params& P, int l, double* f) {
    face_source_fields<KIND>(P.S, P.f, l, f);
  }
  template <typename V, class Fam>
  static __device__ __forceinline__ void pair(const Frame&, const Tgt<V>& t, const V* s, V* acc) {
    const V d0 = t.y0 - s[0], d1 = t.y1 - s[1], d2 = t.y2 - s[2];
    const V e = VT<V>::expneg(sqdist(d0, d1, d2));  // Gaussian data kernel
    if (KIND == LDDMM_DATA_VARIFOLD) {
      const V g = dot3(t.n0, t.n1, t.n2, s[4], s[5], s[6]);
      const V ea = e * s[3];
      acc[0] = fma(ea, g * g, acc[0] + ea);
    } else if (KIND == LDDMM_DATA_MEASURE) {
      acc[0] = fma(e, s[3], acc[0]);
    } else {
      acc[0] = fma(e, s[4], acc[0]);
      acc[1] = fma(e, s[5], acc[1]);
      acc[2] = fma(e, s[6], acc[2]);
    }
  }
  // Expanded-distance form (pairs_kernel_x). Payload: varifold (aw * factor, unit normal), measure
  // (aw * factor), current (fw * surfel * factor). Varifold: 9 FP32 + 1 SFU per pair.
  static constexpr bool kExpand = true;
  static constexpr int NP = (KIND == LDDMM_DATA_VARIFOLD) ? 4 : (KIND == LDDMM_DATA_MEASURE ? 1 : 3);
  template <typename V> struct TgtX { V n0, n1, n2; };
  template <typename V>
  static __device__ __forceinline__ void load_target_x(const Params& P, int i0, int i1, TgtX<V>& t) {
    if (KIND == LDDMM_DATA_VARIFOLD) {
      const FaceRec &r0 = P.T[i0], &r1 = P.T[i1];
      t.n0 = VT<V>::pack(r0.n[0], r1.n[0]);
      t.n1 = VT<V>::pack(r0.n[1], r1.n[1]);
      t.n2 = VT<V>::pack(r0.n[2], r1.n[2]);
    }
  }
  static __device__ __forceinline__ void target_point(const Params& P, int i, double* c) {
    const FaceRec& r = P.T[i];
    c[0] = r.c[0]; c[1] = r.c[1]; c[2] = r.c[2];
  }
  static __device__ __forceinline__ void source_point(const Params& P, int l, double* c, double* f) {
    double fac;
    const FaceRec& r = src_face(P.S, l, fac);
    c[0] = r.c[0]; c[1] = r.c[1]; c[2] = r.c[2];
    if (KIND == LDDMM_DATA_CURRENT) {
      for (int k = 0; k < 3; ++k) f[k] = fac * r.s[k] * r.fw;
    } else {
      f[0] = fac * r.aw;
      if (KIND == LDDMM_DATA_VARIFOLD)
        for (int k = 0; k < 3; ++k) f[1 + k] = r.n[k];
    }
  }
  template <bool X, typename V>
  static __device__ __forceinline__ void accumulate(const TgtX<V>& t, const V*, V e, const V* s, V* acc) {
    const V* w = s + 4;  // the payload of the staged record
    if (KIND == LDDMM_DATA_VARIFOLD) {
      const V g = dot3(t.n0, t.n1, t.n2, w[1], w[2], w[3]);
      acc[0] = fma(e * w[0], fma(g, g, VT<V>::dup(1.0)), acc[0]);
    } else if (KIND == LDDMM_DATA_MEASURE) {
      acc[0] = fma(e, w[0], acc[0]);
    } else {
      acc[0] = fma(e, w[0], acc[0]);
      acc[1] = fma(e, w[1], acc[1]);
      acc[2] = fma(e, w[2], acc[2]);
    }
  }
  static __device__ __forceinline__ void finalize(const Params& P, int i, const double* acc) {
    const FaceRec& r = P.T[i];
    if (KIND == LDDMM_DATA_CURRENT)
      P.dots[i] = r.fw * (r.s[0] * acc[0] + r.s[1] * acc[1] + r.s[2] * acc[2]);
    else
      P.dots[i] = r.aw * acc[0];
  }
};

// ---- gradients: per deformed face z (the vector crossed with the opposite edge), dz (centre term), zw ----
struct FaceGrad {
  double z[3], dz[3], zw, pad;
};

// Varifold gradient pair: z += e aw_l [2g n_l + (1-g^2) n_k] (as Z = sum 2g e aw n_l and W = sum e aw (1-g^2)),
// D = sum e aw (1+g^2) d, S = sum e aw (1+g^2): 22 FP32 + 1 SFU per pair.
template <int KIND>
struct OpSurfGrad {
  static constexpr int NS = 7, NA = (KIND == LDDMM_DATA_VARIFOLD) ? 8 : (KIND == LDDMM_DATA_CURRENT ? 6 : 4);
  static constexpr int kMinCtas = LDDMM_SURFGRAD_MIN_CTAS;
  static constexpr int kUnroll = 8;  // measured 1.9% faster than 4 (varifold, level 6)
  static constexpr bool kCull = true;  // exact culling of far face tiles
  struct Params {
    const FaceRec* T;
    FaceSources S;
    FaceGrad* out;
    Frame f;
  };
  template <typename V> using Tgt = FaceTgt<V>;
  template <typename V>
  static __device__ __forceinline__ void load_target(const Params& P, int i0, int i1, Tgt<V>& t) {
    load_face_target<V, KIND>(P.T, P.f, i0, i1, t);
  }
  static __device__ __forceinline__ void source_fields(const Params& P, int l, double* f) {
    face_source_fields<KIND>(P.S, P.f, l, f);
  }
  template <typename V, class Fam>
  static __device__ __forceinline__ void pair(const Frame&, const Tgt<V>& t, const V* s, V* acc) {
    const V d0 = t.y0 - s[0], d1 = t.y1 - s[1], d2 = t.y2 - s[2];
    const V e = VT<V>::expneg(sqdist(d0, d1, d2));  // Gaussian data kernel
    if (KIND == LDDMM_DATA_VARIFOLD) {
      const V g = dot3(t.n0, t.n1, t.n2, s[4], s[5], s[6]);
      const V ea = e * s[3];
      const V eag = ea * g;
      const V eag2 = eag * g;
      const V t2 = eag + eag;
      acc[0] = fma(t2, s[4], acc[0]);
      acc[1] = fma(t2, s[5], acc[1]);
      acc[2] = fma(t2, s[6], acc[2]);
      acc[3] = acc[3] + (ea - eag2);
      const V eaf = ea + eag2;
      acc[4] = fma(eaf, d0, acc[4]);
      acc[5] = fma(eaf, d1, acc[5]);
      acc[6] = fma(eaf, d2, acc[6]);
      acc[7] = acc[7] + eaf;
    } else if (KIND == LDDMM_DATA_CURRENT) {
      acc[0] = fma(e, s[4], acc[0]);
      acc[1] = fma(e, s[5], acc[1]);
      acc[2] = fma(e, s[6], acc[2]);
      const V ec = e * dot3(t.n0, t.n1, t.n2, s[4], s[5], s[6]);
      acc[3] = fma(ec, d0, acc[3]);
      acc[4] = fma(ec, d1, acc[4]);
      acc[5] = fma(ec, d2, acc[5]);
    } else {
      const V ea = e * s[3];
      acc[0] = acc[0] + ea;
      acc[1] = fma(ea, d0, acc[1]);
      acc[2] = fma(ea, d1, acc[2]);
      acc[3] = fma(ea, d2, acc[3]);
    }
  }
  // Expanded-distance form (pairs_kernel_x; varifold and measure): the centre term sum f (y - x) is written
  // y S - sum f x with S = sum f, a sum these kinds accumulate anyway (varifold: f = e aw (1 + g^2), S in slot 7;
  // measure: f = e aw, slot 0), and the staged X = -2 x gives sum f x = -E/2; no difference y - x is formed
  // (varifold: 19 FP32 + 1 SFU per pair) and no accumulator or staged field is added. Blocks too wide for the form
  // sum f (y - x) directly. Radius^2 bound 32, as for the second-order forward step.
  static constexpr bool kExpand = LDDMM_SURFGRAD_EXPAND != 0 && KIND != LDDMM_DATA_CURRENT;
  static constexpr int NP = (KIND == LDDMM_DATA_VARIFOLD) ? 4 : 1, kRtX = 4;
  static constexpr float kExpandR2 = 32.0f;
  template <typename V> struct TgtX { V n0, n1, n2; };
  template <typename V>
  static __device__ __forceinline__ void load_target_x(const Params& P, int i0, int i1, TgtX<V>& t) {
    if (KIND == LDDMM_DATA_VARIFOLD) {
      const FaceRec &r0 = P.T[i0], &r1 = P.T[i1];
      t.n0 = VT<V>::pack(r0.n[0], r1.n[0]);
      t.n1 = VT<V>::pack(r0.n[1], r1.n[1]);
      t.n2 = VT<V>::pack(r0.n[2], r1.n[2]);
    }
  }
  static __device__ __forceinline__ void target_point(const Params& P, int i, double* c) {
    const FaceRec& r = P.T[i];
    c[0] = r.c[0]; c[1] = r.c[1]; c[2] = r.c[2];
  }
  static __device__ __forceinline__ void source_point(const Params& P, int l, double* c, double* f) {
    double fac;
    const FaceRec& r = src_face(P.S, l, fac);
    c[0] = r.c[0]; c[1] = r.c[1]; c[2] = r.c[2];
    f[0] = fac * r.aw;
    if (KIND == LDDMM_DATA_VARIFOLD)
      for (int k = 0; k < 3; ++k) f[1 + k] = r.n[k];
  }
  // s: staged record (X or x 0-2, |x|^2 3, aw 4, unit normal 5-7)
  template <bool X, typename V>
  static __device__ __forceinline__ void accumulate(const TgtX<V>& t, const V* y, V e, const V* s, V* acc) {
    const V ea = e * s[4];
    if constexpr (KIND == LDDMM_DATA_VARIFOLD) {
      const V g = dot3(t.n0, t.n1, t.n2, s[5], s[6], s[7]);
      const V eag = ea * g;
      const V eag2 = eag * g;
      const V t2 = eag + eag;
      acc[0] = fma(t2, s[5], acc[0]);
      acc[1] = fma(t2, s[6], acc[1]);
      acc[2] = fma(t2, s[7], acc[2]);
      acc[3] = acc[3] + (ea - eag2);
      const V eaf = ea + eag2;
      if constexpr (X) {
        acc[4] = fma(eaf, s[0], acc[4]);
        acc[5] = fma(eaf, s[1], acc[5]);
        acc[6] = fma(eaf, s[2], acc[6]);
      } else {
        acc[4] = fma(eaf, y[0] - s[0], acc[4]);
        acc[5] = fma(eaf, y[1] - s[1], acc[5]);
        acc[6] = fma(eaf, y[2] - s[2], acc[6]);
      }
      acc[7] = acc[7] + eaf;
    } else {
      acc[0] = acc[0] + ea;
      if constexpr (X) {
        acc[1] = fma(ea, s[0], acc[1]);
        acc[2] = fma(ea, s[1], acc[2]);
        acc[3] = fma(ea, s[2], acc[3]);
      } else {
        acc[1] = fma(ea, y[0] - s[0], acc[1]);
        acc[2] = fma(ea, y[1] - s[1], acc[2]);
        acc[3] = fma(ea, y[2] - s[2], acc[3]);
      }
    }
  }
  static __device__ __forceinline__ void x_partial(bool expand, const double* y, const double* v, double* o) {
    for (int c = 0; c < NA; ++c) o[c] = v[c];
    const int d = (KIND == LDDMM_DATA_VARIFOLD) ? 4 : 1, sum = (KIND == LDDMM_DATA_VARIFOLD) ? 7 : 0;
    if (expand)
      for (int c = 0; c < 3; ++c) o[d + c] = y[c] * v[sum] + 0.5 * v[d + c];
  }
  static __device__ __forceinline__ void finalize(const Params& P, int i, const double* acc) {
    const FaceRec& r = P.T[i];
    FaceGrad g;
    const double k23 = -(2.0 / 3.0) * P.f.kappa;
    if (KIND == LDDMM_DATA_VARIFOLD) {
      for (int c = 0; c < 3; ++c) {
        g.z[c] = r.fw * (acc[c] + acc[3] * r.n[c]);
        g.dz[c] = k23 * r.aw * acc[4 + c];
      }
      g.zw = (2.0 / 3.0) * r.fw * r.a * acc[7];
    } else if (KIND == LDDMM_DATA_CURRENT) {
      for (int c = 0; c < 3; ++c) {
        g.z[c] = r.fw * acc[c];
        g.dz[c] = k23 * acc[3 + c];
      }
      g.zw = 0.0;
    } else {
      for (int c = 0; c < 3; ++c) {
        g.z[c] = r.fw * acc[0] * r.n[c];
        g.dz[c] = k23 * r.aw * acc[1 + c];
      }
      g.zw = 0.0;
    }
    g.pad = 0.0;
    P.out[i] = g;
  }
};

// px[v] = sum over incident (face, corner) of dz_f - cross(opposite edge, z_f); pxw[v] = sum zw_f.
__global__ void vertex_gather_kernel(const double* __restrict__ v, const int64_t* __restrict__ faces,
                                     const FaceGrad* __restrict__ g, const int32_t* __restrict__ off,
                                     const int32_t* __restrict__ items, int nv, double* __restrict__ px,
                                     double* __restrict__ pxw) {
  const int vi = blockIdx.x * blockDim.x + threadIdx.x;
  if (vi >= nv) return;
  double acc[3] = {0.0, 0.0, 0.0}, accw = 0.0;
  for (int it = off[vi]; it < off[vi + 1]; ++it) {
    const int item = items[it];
    const int f = item / 3, corner = item - 3 * f;
    const int64_t ia = faces[3 * f + (corner + 1) % 3];
    const int64_t ib = faces[3 * f + (corner + 2) % 3];
    // opposite edge, oriented as in the reference: corner 0 -> x3-x2, 1 -> x1-x3, 2 -> x2-x1 (= x_b - x_a)
    const double e0 = v[3 * ib + 0] - v[3 * ia + 0];
    const double e1 = v[3 * ib + 1] - v[3 * ia + 1];
    const double e2 = v[3 * ib + 2] - v[3 * ia + 2];
    const FaceGrad& G = g[f];
    acc[0] += G.dz[0] - (e1 * G.z[2] - e2 * G.z[1]);
    acc[1] += G.dz[1] - (e2 * G.z[0] - e0 * G.z[2]);
    acc[2] += G.dz[2] - (e0 * G.z[1] - e1 * G.z[0]);
    accw += G.zw;
  }
  px[3 * vi + 0] = acc[0];
  px[3 * vi + 1] = acc[1];
  px[3 * vi + 2] = acc[2];
  if (pxw) pxw[vi] = accw;
}

namespace {

constexpr size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

struct SurfLayout {
  size_t recs, grads, dots, pairs, total;
};

template <typename V, int TPB, int RT>
size_t surf_pairs_bytes(int64_t nf, int64_t nf1) {
  size_t b = 0;
  auto upd = [&](size_t v) { b = v > b ? v : b; };
  upd(pairs_ws_bytes<OpSurfGrad<LDDMM_DATA_VARIFOLD>, V, TPB, RT>(nf, nf + nf1));
  upd(pairs_ws_bytes<OpSurfGrad<LDDMM_DATA_CURRENT>, V, TPB, RT>(nf, nf + nf1));
  upd(pairs_ws_bytes<OpSurfGrad<LDDMM_DATA_MEASURE>, V, TPB, RT>(nf, nf + nf1));
  for (int64_t n : {nf, nf1}) {
    const int64_t m = (n == nf) ? nf + nf1 : nf1;
    upd(pairs_ws_bytes<OpSurfEnergy<LDDMM_DATA_VARIFOLD>, V, TPB, RT>(n, m));
    upd(pairs_ws_bytes<OpSurfEnergy<LDDMM_DATA_CURRENT>, V, TPB, RT>(n, m));
    upd(pairs_ws_bytes<OpSurfEnergy<LDDMM_DATA_MEASURE>, V, TPB, RT>(n, m));
  }
  return b;
}

SurfLayout surf_layout(int64_t nf, int64_t nf1, int precision) {
  SurfLayout L;
  L.recs = 0;
  L.grads = L.recs + align256(sizeof(FaceRec) * (size_t)(nf + nf1));
  L.dots = L.grads + align256(sizeof(FaceGrad) * (size_t)nf);
  L.pairs = L.dots + align256(sizeof(double) * (size_t)(nf > nf1 ? nf : nf1));
  const size_t pb = precision == kFP32Compensated ? surf_pairs_bytes<F2, kTpbLight, kRtLight>(nf, nf1)
                                                  : surf_pairs_bytes<double, kTpb64, kRt64>(nf, nf1);
  L.total = L.pairs + align256(pb);
  return L;
}

template <typename V, int TPB, int RT, int KIND>
int surf_energy(const FaceRec* def, int nf, const FaceRec* tgt, int nf1, const Frame& f, int with_norm0,
                double* energy, double* dots, void* pairs, size_t pairs_bytes, cudaStream_t st) {
  using Op = OpSurfEnergy<KIND>;
  typename Op::Params P;
  P.T = def; P.S = FaceSources{def, nf, tgt, -2.0}; P.dots = dots; P.f = f;
  int rc = run_pairs<Op, V, TPB, RT>(P, nf, (int64_t)nf + nf1, pairs, pairs_bytes, st);
  if (rc != kOk) return rc;
  if (nf > 0) ordered_sum_kernel<<<1, 1024, 0, st>>>(dots, nf, 1.0, energy, 0);
  else if (cudaMemsetAsync(energy, 0, sizeof(double), st) != cudaSuccess) return kCudaError;
  if (with_norm0) {
    P.T = tgt; P.S = FaceSources{tgt, nf1, nullptr, 0.0};
    rc = run_pairs<Op, V, TPB, RT>(P, nf1, nf1, pairs, pairs_bytes, st);
    if (rc != kOk) return rc;
    if (nf1 > 0) ordered_sum_kernel<<<1, 1024, 0, st>>>(dots, nf1, 1.0, energy + 1, 0);
    else if (cudaMemsetAsync(energy + 1, 0, sizeof(double), st) != cudaSuccess) return kCudaError;
  }
  return cudaPeekAtLastError() == cudaSuccess ? kOk : kLaunchFailure;
}

template <typename V, int TPB, int RT, int KIND>
int surf_grad(const FaceRec* def, int nf, const FaceRec* tgt, int nf1, const Frame& f, FaceGrad* grads, void* pairs,
              size_t pairs_bytes, cudaStream_t st) {
  using Op = OpSurfGrad<KIND>;
  typename Op::Params P;
  P.T = def; P.S = FaceSources{def, nf, tgt, -1.0}; P.out = grads; P.f = f;
  return run_pairs<Op, V, TPB, RT>(P, nf, (int64_t)nf + nf1, pairs, pairs_bytes, st);
}

template <int KIND>
int surf_energy_dispatch(int precision, const FaceRec* def, int nf, const FaceRec* tgt, int nf1, const double* origin,
                         double sigma, int with_norm0, double* energy, double* dots, void* pairs, size_t pb,
                         cudaStream_t st) {
  if (precision == kFP32Compensated)
    return surf_energy<F2, kTpbLight, kRtLight, KIND>(def, nf, tgt, nf1, make_frame(origin, sigma, kGauss, true),
                                                      with_norm0, energy, dots, pairs, pb, st);
  return surf_energy<double, kTpb64, kRt64, KIND>(def, nf, tgt, nf1, make_frame(origin, sigma, kGauss, false),
                                                  with_norm0, energy, dots, pairs, pb, st);
}

template <int KIND>
int surf_grad_dispatch(int precision, const FaceRec* def, int nf, const FaceRec* tgt, int nf1, const double* origin,
                       double sigma, FaceGrad* grads, void* pairs, size_t pb, cudaStream_t st) {
  if (precision == kFP32Compensated)
    return surf_grad<F2, kTpbLight, kRtLight, KIND>(def, nf, tgt, nf1, make_frame(origin, sigma, kGauss, true),
                                                    grads, pairs, pb, st);
  return surf_grad<double, kTpb64, kRt64, KIND>(def, nf, tgt, nf1, make_frame(origin, sigma, kGauss, false),
                                                grads, pairs, pb, st);
}

bool bad(const void* p, int64_t n) { return n > 0 && p == nullptr; }

int prep_faces(const double* xdef, const int64_t* faces, int64_t nf, const double* weights, const double* x1,
               const int64_t* faces1, int64_t nf1, const double* weights1, FaceRec* recs, cudaStream_t st) {
  const int b = 256;
  if (nf > 0) face_geometry_kernel<<<(int)((nf + b - 1) / b), b, 0, st>>>(xdef, faces, weights, (int)nf, recs);
  if (nf1 > 0)
    face_geometry_kernel<<<(int)((nf1 + b - 1) / b), b, 0, st>>>(x1, faces1, weights1, (int)nf1, recs + nf);
  return cudaPeekAtLastError() == cudaSuccess ? kOk : kLaunchFailure;
}

}  // namespace

size_t surface_ws_bytes(int64_t nf, int64_t nf1, int precision) { return surf_layout(nf, nf1, precision).total; }

}  // namespace lddmm

using namespace lddmm;

extern "C" {

size_t lddmm_surface_workspace_bytes(int64_t nf, int64_t nf1, int precision) {
  if (nf < 0 || nf1 < 0 || (precision != kFP32Compensated && precision != kFP64)) return 0;
  return surface_ws_bytes(nf, nf1, precision);
}

int lddmm_surface_energy(int kind, const double* xdef, int64_t nv, const int64_t* faces, int64_t nf,
                         const double* weights, const double* x1, int64_t nv1, const int64_t* faces1, int64_t nf1,
                         const double* weights1, double sigma, const double* origin, int with_norm0, double* energy,
                         int precision, void* ws, size_t wsb, lddmm_stream_t stream) {
  if (kind < 0 || kind > 2 || nv < 0 || nf < 0 || nv1 < 0 || nf1 < 0 || bad_sigma(sigma) || bad(xdef, nv) ||
      bad(faces, nf) || bad(x1, nv1) || bad(faces1, nf1) || energy == nullptr)
    return kInvalidArgument;
  if ((nf > 0 && nv == 0) || (nf1 > 0 && nv1 == 0)) return kInvalidArgument;
  if (nf > INT32_MAX / 8 || nf1 > INT32_MAX / 8) return kInvalidArgument;
  if (precision != kFP32Compensated && precision != kFP64) return kInvalidArgument;
  const SurfLayout L = surf_layout(nf, nf1, precision);
  if (ws == nullptr || wsb < L.total) return kWorkspaceTooSmall;
  cudaStream_t st = (cudaStream_t)stream;
  char* base = reinterpret_cast<char*>(ws);
  FaceRec* recs = reinterpret_cast<FaceRec*>(base + L.recs);
  double* dots = reinterpret_cast<double*>(base + L.dots);
  int rc = prep_faces(xdef, faces, nf, weights, x1, faces1, nf1, weights1, recs, st);
  if (rc != kOk) return rc;
  const size_t pb = wsb - L.pairs;
  void* pairs = base + L.pairs;
  if (kind == LDDMM_DATA_VARIFOLD)
    return surf_energy_dispatch<LDDMM_DATA_VARIFOLD>(precision, recs, (int)nf, recs + nf, (int)nf1, origin, sigma,
                                                     with_norm0, energy, dots, pairs, pb, st);
  if (kind == LDDMM_DATA_CURRENT)
    return surf_energy_dispatch<LDDMM_DATA_CURRENT>(precision, recs, (int)nf, recs + nf, (int)nf1, origin, sigma,
                                                    with_norm0, energy, dots, pairs, pb, st);
  return surf_energy_dispatch<LDDMM_DATA_MEASURE>(precision, recs, (int)nf, recs + nf, (int)nf1, origin, sigma,
                                                  with_norm0, energy, dots, pairs, pb, st);
}

int lddmm_surface_gradient(int kind, const double* xdef, int64_t nv, const int64_t* faces, int64_t nf,
                           const double* weights, const int32_t* vf_offsets, const int32_t* vf_items,
                           const double* x1, int64_t nv1, const int64_t* faces1, int64_t nf1, const double* weights1,
                           double sigma, const double* origin, double* px, double* pxw, int precision, void* ws,
                           size_t wsb, lddmm_stream_t stream) {
  if (kind < 0 || kind > 2 || nv < 0 || nf < 0 || nv1 < 0 || nf1 < 0 || bad_sigma(sigma) || bad(xdef, nv) ||
      bad(faces, nf) || bad(x1, nv1) || bad(faces1, nf1) || bad(px, nv) || vf_offsets == nullptr ||
      bad(vf_items, nf))
    return kInvalidArgument;
  if ((nf > 0 && nv == 0) || (nf1 > 0 && nv1 == 0)) return kInvalidArgument;
  if (nf > INT32_MAX / 8 || nf1 > INT32_MAX / 8 || nv > INT32_MAX / 8) return kInvalidArgument;
  if (pxw != nullptr && kind != LDDMM_DATA_VARIFOLD) return kUnsupported;
  if (precision != kFP32Compensated && precision != kFP64) return kInvalidArgument;
  const SurfLayout L = surf_layout(nf, nf1, precision);
  if (ws == nullptr || wsb < L.total) return kWorkspaceTooSmall;
  if (nv == 0) return kOk;
  cudaStream_t st = (cudaStream_t)stream;
  char* base = reinterpret_cast<char*>(ws);
  FaceRec* recs = reinterpret_cast<FaceRec*>(base + L.recs);
  FaceGrad* grads = reinterpret_cast<FaceGrad*>(base + L.grads);
  int rc = prep_faces(xdef, faces, nf, weights, x1, faces1, nf1, weights1, recs, st);
  if (rc != kOk) return rc;
  const size_t pb = wsb - L.pairs;
  void* pairs = base + L.pairs;
  if (kind == LDDMM_DATA_VARIFOLD)
    rc = surf_grad_dispatch<LDDMM_DATA_VARIFOLD>(precision, recs, (int)nf, recs + nf, (int)nf1, origin, sigma, grads,
                                                 pairs, pb, st);
  else if (kind == LDDMM_DATA_CURRENT)
    rc = surf_grad_dispatch<LDDMM_DATA_CURRENT>(precision, recs, (int)nf, recs + nf, (int)nf1, origin, sigma, grads,
                                                pairs, pb, st);
  else
    rc = surf_grad_dispatch<LDDMM_DATA_MEASURE>(precision, recs, (int)nf, recs + nf, (int)nf1, origin, sigma, grads,
                                                pairs, pb, st);
  if (rc != kOk) return rc;
  const int b = 256;
  vertex_gather_kernel<<<(int)((nv + b - 1) / b), b, 0, st>>>(xdef, faces, grads, vf_offsets, vf_items, (int)nv, px,
                                                              pxw);
  return cudaPeekAtLastError() == cudaSuccess ? kOk : kLaunchFailure;
}

int lddmm_vertex_face_table(const int64_t* faces, int64_t nf, int64_t nv, int32_t* off, int32_t* items) {
  if (nf < 0 || nv < 0 || (nf > 0 && (faces == nullptr || items == nullptr)) || off == nullptr) return kInvalidArgument;
  if (3 * nf > INT32_MAX) return kInvalidArgument;
  std::vector<int32_t> cnt((size_t)nv + 1, 0);
  for (int64_t i = 0; i < 3 * nf; ++i) {
    const int64_t v = faces[i];
    if (v < 0 || v >= nv) return kInvalidArgument;
    cnt[(size_t)v + 1]++;
  }
  off[0] = 0;
  for (int64_t v = 0; v < nv; ++v) off[v + 1] = off[v] + cnt[(size_t)v + 1];
  std::vector<int32_t> pos(off, off + nv);
  for (int64_t i = 0; i < 3 * nf; ++i) items[pos[(size_t)faces[i]]++] = (int32_t)i;
  return kOk;
}

}  // extern "C"
