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

template <typename R>
__device__ __forceinline__ void face_point(const FaceRec& r, const Frame& f, R& a, R& b, R& c) {
  a = (R)((r.c[0] - f.o0) * f.s);
  b = (R)((r.c[1] - f.o1) * f.s);
  c = (R)((r.c[2] - f.o2) * f.s);
}

// Source record: (c', aw * factor) and the unit normal, or (c') and the weighted surfel * factor (current).
template <typename R, int KIND>
__device__ __forceinline__ void load_face_source(const FaceSources& S, const Frame& f, int l, V4<R>* s) {
  double fac;
  const FaceRec& r = src_face(S, l, fac);
  face_point(r, f, s[0].x, s[0].y, s[0].z);
  if (KIND == LDDMM_DATA_CURRENT) {
    s[0].w = R(0);
    s[1].x = (R)(fac * r.s[0] * r.fw);
    s[1].y = (R)(fac * r.s[1] * r.fw);
    s[1].z = (R)(fac * r.s[2] * r.fw);
  } else {
    s[0].w = (R)(fac * r.aw);
    s[1].x = (R)r.n[0];
    s[1].y = (R)r.n[1];
    s[1].z = (R)r.n[2];
  }
  s[1].w = R(0);
}

// ---- energies: dots[k] = weight_k * sum_l e_kl payload_kl ----
template <typename R, int KIND>
struct OpSurfEnergy {
  static constexpr int NV = 2, NA = (KIND == LDDMM_DATA_CURRENT) ? 3 : 1;
  struct Params {
    const FaceRec* T;
    FaceSources S;
    double* dots;
    Frame f;
  };
  struct Tgt { R y0, y1, y2, n0, n1, n2; };
  static __device__ __forceinline__ void load_target(const Params& P, int i, Tgt& t) {
    const FaceRec& r = P.T[i];
    face_point(r, P.f, t.y0, t.y1, t.y2);
    t.n0 = (R)r.n[0]; t.n1 = (R)r.n[1]; t.n2 = (R)r.n[2];
  }
  static __device__ __forceinline__ void load_source(const Params& P, int l, V4<R>* s) {
    load_face_source<R, KIND>(P.S, P.f, l, s);
  }
  static __device__ __forceinline__ void pair(const Tgt& t, const V4<R>* s, R* acc) {
    const R d0 = t.y0 - s[0].x, d1 = t.y1 - s[0].y, d2 = t.y2 - s[0].z;
    const R e = PT<R>::expneg(d0 * d0 + d1 * d1 + d2 * d2);
    if (KIND == LDDMM_DATA_VARIFOLD) {
      const R g = t.n0 * s[1].x + t.n1 * s[1].y + t.n2 * s[1].z;
      acc[0] += (e * s[0].w) * (R(1) + g * g);
    } else if (KIND == LDDMM_DATA_MEASURE) {
      acc[0] += e * s[0].w;
    } else {
      acc[0] += e * s[1].x;
      acc[1] += e * s[1].y;
      acc[2] += e * s[1].z;
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

template <typename R, int KIND>
struct OpSurfGrad {
  static constexpr int NV = 2, NA = (KIND == LDDMM_DATA_VARIFOLD) ? 8 : (KIND == LDDMM_DATA_CURRENT ? 6 : 4);
  struct Params {
    const FaceRec* T;
    FaceSources S;
    FaceGrad* out;
    Frame f;
  };
  struct Tgt { R y0, y1, y2, n0, n1, n2; };
  static __device__ __forceinline__ void load_target(const Params& P, int i, Tgt& t) {
    const FaceRec& r = P.T[i];
    face_point(r, P.f, t.y0, t.y1, t.y2);
    if (KIND == LDDMM_DATA_CURRENT) {
      t.n0 = (R)(r.s[0] * r.fw); t.n1 = (R)(r.s[1] * r.fw); t.n2 = (R)(r.s[2] * r.fw);
    } else {
      t.n0 = (R)r.n[0]; t.n1 = (R)r.n[1]; t.n2 = (R)r.n[2];
    }
  }
  static __device__ __forceinline__ void load_source(const Params& P, int l, V4<R>* s) {
    load_face_source<R, KIND>(P.S, P.f, l, s);
  }
  static __device__ __forceinline__ void pair(const Tgt& t, const V4<R>* s, R* acc) {
    const R d0 = t.y0 - s[0].x, d1 = t.y1 - s[0].y, d2 = t.y2 - s[0].z;
    const R e = PT<R>::expneg(d0 * d0 + d1 * d1 + d2 * d2);
    if (KIND == LDDMM_DATA_VARIFOLD) {
      // z: sum e aw_l [2g n_l + (1-g^2) n_k]; d: sum e aw_l (1+g^2) d; sw: sum e aw_l (1+g^2)
      const R g = t.n0 * s[1].x + t.n1 * s[1].y + t.n2 * s[1].z;
      const R ea = e * s[0].w;
      const R f = R(1) + g * g;
      const R t2 = R(2) * g * ea;
      acc[0] += t2 * s[1].x;
      acc[1] += t2 * s[1].y;
      acc[2] += t2 * s[1].z;
      acc[3] += ea * (R(1) - g * g);
      const R eaf = ea * f;
      acc[4] += eaf * d0;
      acc[5] += eaf * d1;
      acc[6] += eaf * d2;
      acc[7] += eaf;
    } else if (KIND == LDDMM_DATA_CURRENT) {
      acc[0] += e * s[1].x;
      acc[1] += e * s[1].y;
      acc[2] += e * s[1].z;
      const R ec = e * (t.n0 * s[1].x + t.n1 * s[1].y + t.n2 * s[1].z);
      acc[3] += ec * d0;
      acc[4] += ec * d1;
      acc[5] += ec * d2;
    } else {
      const R ea = e * s[0].w;
      acc[0] += ea;
      acc[1] += ea * d0;
      acc[2] += ea * d1;
      acc[3] += ea * d2;
    }
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

template <typename R, int TPB, int RT>
size_t surf_pairs_bytes(int64_t nf, int64_t nf1) {
  size_t b = 0;
  auto upd = [&](size_t v) { b = v > b ? v : b; };
  upd(pairs_ws_bytes<OpSurfGrad<R, LDDMM_DATA_VARIFOLD>, R, TPB, RT>(nf, nf + nf1, kCtasPerSm));
  upd(pairs_ws_bytes<OpSurfEnergy<R, LDDMM_DATA_CURRENT>, R, TPB, RT>(nf, nf + nf1, kCtasPerSm));
  upd(pairs_ws_bytes<OpSurfEnergy<R, LDDMM_DATA_CURRENT>, R, TPB, RT>(nf1, nf1, kCtasPerSm));
  upd(pairs_ws_bytes<OpSurfGrad<R, LDDMM_DATA_CURRENT>, R, TPB, RT>(nf, nf + nf1, kCtasPerSm));
  return b;
}

SurfLayout surf_layout(int64_t nf, int64_t nf1, int precision) {
  SurfLayout L;
  L.recs = 0;
  L.grads = L.recs + align256(sizeof(FaceRec) * (size_t)(nf + nf1));
  L.dots = L.grads + align256(sizeof(FaceGrad) * (size_t)nf);
  L.pairs = L.dots + align256(sizeof(double) * (size_t)(nf > nf1 ? nf : nf1));
  const size_t pb = precision == kFP32Compensated ? surf_pairs_bytes<float, kTpbLight, kRtLight>(nf, nf1)
                                                  : surf_pairs_bytes<double, kTpb64, kRt64>(nf, nf1);
  L.total = L.pairs + align256(pb);
  return L;
}

template <typename R, int TPB, int RT, int KIND>
int surf_energy(const FaceRec* def, int nf, const FaceRec* tgt, int nf1, const Frame& f, int with_norm0,
                double* energy, double* dots, void* pairs, size_t pairs_bytes, cudaStream_t st) {
  using Op = OpSurfEnergy<R, KIND>;
  typename Op::Params P;
  P.T = def; P.S = FaceSources{def, nf, tgt, -2.0}; P.dots = dots; P.f = f;
  int rc = run_pairs<Op, R, TPB, RT>(P, nf, (int64_t)nf + nf1, pairs, pairs_bytes, st, kCtasPerSm);
  if (rc != kOk) return rc;
  if (nf > 0) ordered_sum_kernel<<<1, 1024, 0, st>>>(dots, nf, 1.0, energy, 0);
  else if (cudaMemsetAsync(energy, 0, sizeof(double), st) != cudaSuccess) return kCudaError;
  if (with_norm0) {
    P.T = tgt; P.S = FaceSources{tgt, nf1, nullptr, 0.0};
    rc = run_pairs<Op, R, TPB, RT>(P, nf1, nf1, pairs, pairs_bytes, st, kCtasPerSm);
    if (rc != kOk) return rc;
    if (nf1 > 0) ordered_sum_kernel<<<1, 1024, 0, st>>>(dots, nf1, 1.0, energy + 1, 0);
    else if (cudaMemsetAsync(energy + 1, 0, sizeof(double), st) != cudaSuccess) return kCudaError;
  }
  return cudaPeekAtLastError() == cudaSuccess ? kOk : kLaunchFailure;
}

template <typename R, int TPB, int RT, int KIND>
int surf_grad(const FaceRec* def, int nf, const FaceRec* tgt, int nf1, const Frame& f, FaceGrad* grads, void* pairs,
              size_t pairs_bytes, cudaStream_t st) {
  using Op = OpSurfGrad<R, KIND>;
  typename Op::Params P;
  P.T = def; P.S = FaceSources{def, nf, tgt, -1.0}; P.out = grads; P.f = f;
  return run_pairs<Op, R, TPB, RT>(P, nf, (int64_t)nf + nf1, pairs, pairs_bytes, st, kCtasPerSm);
}

template <int KIND>
int surf_energy_dispatch(int precision, const FaceRec* def, int nf, const FaceRec* tgt, int nf1, const double* origin,
                         double sigma, int with_norm0, double* energy, double* dots, void* pairs, size_t pb,
                         cudaStream_t st) {
  if (precision == kFP32Compensated)
    return surf_energy<float, kTpbLight, kRtLight, KIND>(def, nf, tgt, nf1, make_frame(origin, sigma, PT<float>::kScale),
                                                         with_norm0, energy, dots, pairs, pb, st);
  return surf_energy<double, kTpb64, kRt64, KIND>(def, nf, tgt, nf1, make_frame(origin, sigma, PT<double>::kScale),
                                                  with_norm0, energy, dots, pairs, pb, st);
}

template <int KIND>
int surf_grad_dispatch(int precision, const FaceRec* def, int nf, const FaceRec* tgt, int nf1, const double* origin,
                       double sigma, FaceGrad* grads, void* pairs, size_t pb, cudaStream_t st) {
  if (precision == kFP32Compensated)
    return surf_grad<float, kTpbLight, kRtLight, KIND>(def, nf, tgt, nf1, make_frame(origin, sigma, PT<float>::kScale),
                                                       grads, pairs, pb, st);
  return surf_grad<double, kTpb64, kRt64, KIND>(def, nf, tgt, nf1, make_frame(origin, sigma, PT<double>::kScale),
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
