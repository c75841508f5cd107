// Landmark shooting and its adjoint: fused step kernels (one exp per pair shared by every sum of a step)
// with the FP64 state update done in the epilogue. Replaces base/pointEvolution.py.
#include "../../include/lddmm_b200.h"
#include "kernel_ops.cuh"
#include "launch_config.cuh"

namespace lddmm {

// Second-order forward step (secondOrderEvolution loop body, base/pointEvolution.py:433-449):
//   x1 = x + dt K(x) a,   a1 = a + dt za with za = -DK^T(x; a, a) = kappa sum_l e (a_k.a_l) d.
// Accumulators: X = sum e a_l (3), A = sum e (a_k.a_l) d (3). 16 FP32 + 1 SFU per pair.
template <typename R>
struct OpSOFwd {
  static constexpr int NV = 2, NA = 6;
  struct Params {
    const double *x, *a;
    double *x1, *a1;
    Frame f;
    double dt;
  };
  struct Tgt { R y0, y1, y2, a0, a1, a2; };
  static __device__ __forceinline__ void load_target(const Params& P, int i, Tgt& t) {
    load_point(P.x, i, P.f, t.y0, t.y1, t.y2);
    load_vec(P.a, i, t.a0, t.a1, t.a2);
  }
  static __device__ __forceinline__ void load_source(const Params& P, int l, V4<R>* s) {
    load_point(P.x, l, P.f, s[0].x, s[0].y, s[0].z);
    load_vec(P.a, l, s[1].x, s[1].y, s[1].z);
    s[0].w = s[1].w = R(0);
  }
  static __device__ __forceinline__ void pair(const Tgt& t, const V4<R>* s, R* acc) {
    const R d0 = t.y0 - s[0].x, d1 = t.y1 - s[0].y, d2 = t.y2 - s[0].z;
    const R e = PT<R>::expneg(d0 * d0 + d1 * d1 + d2 * d2);
    acc[0] += e * s[1].x;
    acc[1] += e * s[1].y;
    acc[2] += e * s[1].z;
    const R ec = e * (t.a0 * s[1].x + t.a1 * s[1].y + t.a2 * s[1].z);
    acc[3] += ec * d0;
    acc[4] += ec * d1;
    acc[5] += ec * d2;
  }
  static __device__ __forceinline__ void finalize(const Params& P, int i, const double* acc) {
    const double ka = P.dt * P.f.kappa;
    for (int c = 0; c < 3; ++c) {
      P.x1[3 * i + c] = P.x[3 * i + c] + P.dt * acc[c];
      P.a1[3 * i + c] = P.a[3 * i + c] + ka * acc[3 + c];
    }
  }
};

// Second-order adjoint step (secondOrderCovector loop body, base/pointEvolution.py:539-546):
//   zpx = DK^T_sym(x; px, a) - DDK11and12(x; a, a, pa),   zpa = K(x) px - DK1and2(x; pa, a)
//   px_prev = px + dt zpx,  pa_prev = pa + dt zpa.
// With c1' = px'_k.a_l + a_k.px'_l (px' = -kappa px), c2'' = a''_k.a_l (a'' = -kappa^2 a), q = dpa = pa_k - pa_l,
// dq = d.q the accumulators are
//   G = sum e (c1' + c2'' dq) d (3), C = sum e c2'' (1), D = sum e c2'' pa_l (3), E = sum e px'_l (3),
//   F = sum e dq a_l (3)
// and zpx = G + (pa_k C - D)/(sigma^2 (-kappa^2)), zpa = E/(-kappa) + kappa F. 38 FP32 + 1 SFU per pair.
template <typename R>
struct OpSOBwd {
  static constexpr int NV = 3, NA = 13;
  struct Params {
    const double *x, *a, *px, *pa;
    double *px_prev, *pa_prev;
    Frame f;
    double dt;
  };
  struct Tgt { R y0, y1, y2, a0, a1, a2, b0, b1, b2, p0, p1, p2, q0, q1, q2; };
  static __device__ __forceinline__ void load_target(const Params& P, int i, Tgt& t) {
    const double k = P.f.kappa;
    load_point(P.x, i, P.f, t.y0, t.y1, t.y2);
    load_vec(P.a, i, t.a0, t.a1, t.a2);
    t.b0 = (R)(-k * k * P.a[3 * i + 0]);
    t.b1 = (R)(-k * k * P.a[3 * i + 1]);
    t.b2 = (R)(-k * k * P.a[3 * i + 2]);
    t.p0 = (R)(-k * P.px[3 * i + 0]);
    t.p1 = (R)(-k * P.px[3 * i + 1]);
    t.p2 = (R)(-k * P.px[3 * i + 2]);
    load_vec(P.pa, i, t.q0, t.q1, t.q2);
  }
  static __device__ __forceinline__ void load_source(const Params& P, int l, V4<R>* s) {
    const double k = P.f.kappa;
    load_point(P.x, l, P.f, s[0].x, s[0].y, s[0].z);
    load_vec(P.a, l, s[1].x, s[1].y, s[1].z);
    load_vec(P.pa, l, s[2].x, s[2].y, s[2].z);
    s[0].w = (R)(-k * P.px[3 * l + 0]);
    s[1].w = (R)(-k * P.px[3 * l + 1]);
    s[2].w = (R)(-k * P.px[3 * l + 2]);
  }
  static __device__ __forceinline__ void pair(const Tgt& t, const V4<R>* s, R* acc) {
    const R d0 = t.y0 - s[0].x, d1 = t.y1 - s[0].y, d2 = t.y2 - s[0].z;
    const R e = PT<R>::expneg(d0 * d0 + d1 * d1 + d2 * d2);
    const R dq = d0 * (t.q0 - s[2].x) + d1 * (t.q1 - s[2].y) + d2 * (t.q2 - s[2].z);
    const R c1 = t.p0 * s[1].x + t.p1 * s[1].y + t.p2 * s[1].z + t.a0 * s[0].w + t.a1 * s[1].w + t.a2 * s[2].w;
    const R c2 = t.b0 * s[1].x + t.b1 * s[1].y + t.b2 * s[1].z;
    const R eg = e * (c1 + c2 * dq);
    acc[0] += eg * d0;
    acc[1] += eg * d1;
    acc[2] += eg * d2;
    const R ec2 = e * c2;
    acc[3] += ec2;
    acc[4] += ec2 * s[2].x;
    acc[5] += ec2 * s[2].y;
    acc[6] += ec2 * s[2].z;
    acc[7] += e * s[0].w;
    acc[8] += e * s[1].w;
    acc[9] += e * s[2].w;
    const R edq = e * dq;
    acc[10] += edq * s[1].x;
    acc[11] += edq * s[1].y;
    acc[12] += edq * s[1].z;
  }
  static __device__ __forceinline__ void finalize(const Params& P, int i, const double* acc) {
    const double k = P.f.kappa;
    const double cd = -1.0 / (k * k) * P.f.inv_s2;  // converts the c2''-weighted sums back, times 1/sigma^2
    for (int c = 0; c < 3; ++c) {
      const double pa = P.pa[3 * i + c];
      const double zpx = acc[c] + cd * (pa * acc[3] - acc[4 + c]);
      const double zpa = -acc[7 + c] / k + k * acc[10 + c];
      P.px_prev[3 * i + c] = P.px[3 * i + c] + P.dt * zpx;
      P.pa_prev[3 * i + c] = pa + P.dt * zpa;
    }
  }
};

// First-order adjoint step with the gradient of the same step (base/pointEvolution.py:186-201, :221-223;
// base/surfaceMatching.py:810, :879-891):
//   p_t = p_{t+1} + dt DK^T_lddmm(x_t; p_{t+1}, a_t) = p_{t+1} - dt kappa sum_l e (p_k.a_l + a_k.q_l) d,
//   q_l = p_l - 2 w a_l;  dat_t = K(x_t)(2 w a_t - p_{t+1}) = -sum_l e q_l (euclidean) or 2 w a_t - p_{t+1}.
// Accumulators: A = sum e c d (3), Q = sum e q_l (3). 19 FP32 + 1 SFU per pair.
template <typename R>
struct OpFOBwd {
  static constexpr int NV = 3, NA = 6;
  struct Params {
    const double *x, *a, *p;
    double *p_prev, *dat;
    Frame f;
    double dt, w;
    int euclidean;
  };
  struct Tgt { R y0, y1, y2, p0, p1, p2, a0, a1, a2; };
  static __device__ __forceinline__ void load_target(const Params& P, int i, Tgt& t) {
    load_point(P.x, i, P.f, t.y0, t.y1, t.y2);
    load_vec(P.p, i, t.p0, t.p1, t.p2);
    load_vec(P.a, i, t.a0, t.a1, t.a2);
  }
  static __device__ __forceinline__ void load_source(const Params& P, int l, V4<R>* s) {
    load_point(P.x, l, P.f, s[0].x, s[0].y, s[0].z);
    load_vec(P.a, l, s[1].x, s[1].y, s[1].z);
    for (int c = 0; c < 3; ++c) {
      const R q = (R)(P.p[3 * l + c] - 2.0 * P.w * P.a[3 * l + c]);
      if (c == 0) s[2].x = q; else if (c == 1) s[2].y = q; else s[2].z = q;
    }
    s[0].w = s[1].w = s[2].w = R(0);
  }
  static __device__ __forceinline__ void pair(const Tgt& t, const V4<R>* s, R* acc) {
    const R d0 = t.y0 - s[0].x, d1 = t.y1 - s[0].y, d2 = t.y2 - s[0].z;
    const R e = PT<R>::expneg(d0 * d0 + d1 * d1 + d2 * d2);
    const R c = t.p0 * s[1].x + t.p1 * s[1].y + t.p2 * s[1].z + t.a0 * s[2].x + t.a1 * s[2].y + t.a2 * s[2].z;
    const R ec = e * c;
    acc[0] += ec * d0;
    acc[1] += ec * d1;
    acc[2] += ec * d2;
    acc[3] += e * s[2].x;
    acc[4] += e * s[2].y;
    acc[5] += e * s[2].z;
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

size_t shooting_ws_bytes(int64_t n, int precision) {
  size_t b = 0;
  auto upd = [&](size_t v) { b = v > b ? v : b; };
  if (precision == kFP32Compensated) {
    upd(pairs_ws_bytes<OpSOFwd<float>, float, kTpbLight, kRtLight>(n, n, kCtasPerSm));
    upd(pairs_ws_bytes<OpSOBwd<float>, float, kTpbHeavy, kRtHeavy>(n, n, kCtasPerSm));
    upd(pairs_ws_bytes<OpFOBwd<float>, float, kTpbLight, kRtLight>(n, n, kCtasPerSm));
    upd(pairs_ws_bytes<OpK<float>, float, kTpbLight, kRtLight>(n, n, kCtasPerSm));
  } else {
    upd(pairs_ws_bytes<OpSOBwd<double>, double, kTpb64, kRt64>(n, n, kCtasPerSm));
    upd(pairs_ws_bytes<OpK<double>, double, kTpb64, kRt64>(n, n, kCtasPerSm));
  }
  // per-point dot products for the FP64 energy reductions live after the pair partials
  return b + (size_t)(n > 0 ? n : 0) * sizeof(double) + 256;
}

namespace {

inline double* dots_region(void* ws, size_t pair_bytes) {
  size_t off = (pair_bytes + 255) & ~(size_t)255;
  return reinterpret_cast<double*>(reinterpret_cast<char*>(ws) + off);
}

template <typename R, int TPB, int RT>
int k_energy_and_update(const double* x, const double* a, int64_t n, const Frame& f, const double* base,
                        double base_sign, double scale, double* out, const double* dotw, double* energy,
                        double escale, int accumulate, void* ws, size_t wsb, cudaStream_t st) {
  typename OpK<R>::Params P;
  P.y = x; P.x = x; P.a = a; P.out = out; P.f = f;
  P.base = base; P.base_sign = base_sign; P.scale = scale;
  const size_t pb = pairs_ws_bytes<OpK<R>, R, TPB, RT>(n, n, kCtasPerSm);
  if (energy) {
    if (((pb + 255) & ~(size_t)255) + (size_t)n * sizeof(double) > wsb) return kWorkspaceTooSmall;
    P.dotw = dotw;
    P.dots = dots_region(ws, pb);
  }
  int rc = run_pairs<OpK<R>, R, TPB, RT>(P, n, n, ws, wsb, st, kCtasPerSm);
  if (rc != kOk) return rc;
  if (energy) {
    ordered_sum_kernel<<<1, 1024, 0, st>>>(P.dots, (int)n, escale, energy, accumulate);
    if (cudaPeekAtLastError() != cudaSuccess) return kLaunchFailure;
  }
  return kOk;
}

template <typename R, int TPB, int RT, int TPBH, int RTH>
int so_shoot(const double* x0, const double* a0, int64_t n, int64_t T, const Frame& f, double dt, double* xt,
             double* at, void* ws, size_t wsb, cudaStream_t st) {
  const size_t stride = (size_t)n * 3;
  if (cudaMemcpyAsync(xt, x0, stride * sizeof(double), cudaMemcpyDeviceToDevice, st) != cudaSuccess) return kCudaError;
  if (cudaMemcpyAsync(at, a0, stride * sizeof(double), cudaMemcpyDeviceToDevice, st) != cudaSuccess) return kCudaError;
  for (int64_t t = 0; t < T; ++t) {
    typename OpSOFwd<R>::Params P;
    P.x = xt + t * stride; P.a = at + t * stride;
    P.x1 = xt + (t + 1) * stride; P.a1 = at + (t + 1) * stride;
    P.f = f; P.dt = dt;
    int rc = run_pairs<OpSOFwd<R>, R, TPB, RT>(P, n, n, ws, wsb, st, kCtasPerSm);
    if (rc != kOk) return rc;
  }
  return kOk;
}

template <typename R, int TPB, int RT, int TPBH, int RTH>
int so_gradient(const double* xt, const double* at, int64_t n, int64_t T, const Frame& f, double dt,
                const double* px1, const double* pa1, double* pxt, double* pat, double* da0, void* ws, size_t wsb,
                cudaStream_t st) {
  const size_t stride = (size_t)n * 3;
  if (cudaMemcpyAsync(pxt + T * stride, px1, stride * sizeof(double), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    return kCudaError;
  if (cudaMemcpyAsync(pat + T * stride, pa1, stride * sizeof(double), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    return kCudaError;
  for (int64_t t = T - 1; t >= 0; --t) {
    typename OpSOBwd<R>::Params P;
    P.x = xt + t * stride; P.a = at + t * stride;
    P.px = pxt + (t + 1) * stride; P.pa = pat + (t + 1) * stride;
    P.px_prev = pxt + t * stride; P.pa_prev = pat + t * stride;
    P.f = f; P.dt = dt;
    int rc = run_pairs<OpSOBwd<R>, R, TPBH, RTH>(P, n, n, ws, wsb, st, kCtasPerSm);
    if (rc != kOk) return rc;
  }
  if (da0)
    return k_energy_and_update<R, TPB, RT>(xt, at, n, f, pat, -1.0, 1.0, da0, nullptr, nullptr, 0.0, 0, ws, wsb, st);
  return kOk;
}

bool bad(const void* p, int64_t n) { return n > 0 && p == nullptr; }

}  // namespace
}  // namespace lddmm

using namespace lddmm;

extern "C" {

int lddmm_second_order_step(const double* x, const double* a, int64_t n, double sigma, double dt,
                            const double* origin, double* x_next, double* a_next, int precision, void* ws,
                            size_t wsb, lddmm_stream_t stream) {
  if (n < 0 || bad_sigma(sigma) || bad(x, n) || bad(a, n) || bad(x_next, n) || bad(a_next, n)) return kInvalidArgument;
  cudaStream_t st = (cudaStream_t)stream;
  if (precision == kFP32Compensated) {
    OpSOFwd<float>::Params P{x, a, x_next, a_next, make_frame(origin, sigma, PT<float>::kScale), dt};
    return run_pairs<OpSOFwd<float>, float, kTpbLight, kRtLight>(P, n, n, ws, wsb, st, kCtasPerSm);
  }
  if (precision == kFP64) {
    OpSOFwd<double>::Params P{x, a, x_next, a_next, make_frame(origin, sigma, PT<double>::kScale), dt};
    return run_pairs<OpSOFwd<double>, double, kTpb64, kRt64>(P, n, n, ws, wsb, st, kCtasPerSm);
  }
  return kInvalidArgument;
}

int lddmm_second_order_shoot(const double* x0, const double* a0, int64_t n, int64_t T, double sigma, double dt,
                             const double* origin, double* xt, double* at, int precision, void* ws, size_t wsb,
                             lddmm_stream_t stream) {
  if (n < 0 || T < 0 || bad_sigma(sigma) || bad(x0, n) || bad(a0, n) || bad(xt, n) || bad(at, n)) return kInvalidArgument;
  if (n == 0) return kOk;
  cudaStream_t st = (cudaStream_t)stream;
  if (precision == kFP32Compensated)
    return so_shoot<float, kTpbLight, kRtLight, kTpbHeavy, kRtHeavy>(
        x0, a0, n, T, make_frame(origin, sigma, PT<float>::kScale), dt, xt, at, ws, wsb, st);
  if (precision == kFP64)
    return so_shoot<double, kTpb64, kRt64, kTpb64, kRt64>(x0, a0, n, T, make_frame(origin, sigma, PT<double>::kScale),
                                                          dt, xt, at, ws, wsb, st);
  return kInvalidArgument;
}

int lddmm_second_order_adjoint_step(const double* x, const double* a, const double* px, const double* pa, int64_t n,
                                    double sigma, double dt, const double* origin, double* px_prev, double* pa_prev,
                                    int precision, void* ws, size_t wsb, lddmm_stream_t stream) {
  if (n < 0 || bad_sigma(sigma) || bad(x, n) || bad(a, n) || bad(px, n) || bad(pa, n) || bad(px_prev, n) ||
      bad(pa_prev, n))
    return kInvalidArgument;
  cudaStream_t st = (cudaStream_t)stream;
  if (precision == kFP32Compensated) {
    OpSOBwd<float>::Params P{x, a, px, pa, px_prev, pa_prev, make_frame(origin, sigma, PT<float>::kScale), dt};
    return run_pairs<OpSOBwd<float>, float, kTpbHeavy, kRtHeavy>(P, n, n, ws, wsb, st, kCtasPerSm);
  }
  if (precision == kFP64) {
    OpSOBwd<double>::Params P{x, a, px, pa, px_prev, pa_prev, make_frame(origin, sigma, PT<double>::kScale), dt};
    return run_pairs<OpSOBwd<double>, double, kTpb64, kRt64>(P, n, n, ws, wsb, st, kCtasPerSm);
  }
  return kInvalidArgument;
}

int lddmm_second_order_gradient(const double* xt, const double* at, int64_t n, int64_t T, double sigma, double dt,
                                const double* px1, const double* pa1, const double* origin, double* pxt, double* pat,
                                double* da0, int precision, void* ws, size_t wsb, lddmm_stream_t stream) {
  if (n < 0 || T < 0 || bad_sigma(sigma) || bad(xt, n) || bad(at, n) || bad(px1, n) || bad(pa1, n) || bad(pxt, n) ||
      bad(pat, n))
    return kInvalidArgument;
  if (n == 0) return kOk;
  cudaStream_t st = (cudaStream_t)stream;
  if (precision == kFP32Compensated)
    return so_gradient<float, kTpbLight, kRtLight, kTpbHeavy, kRtHeavy>(
        xt, at, n, T, make_frame(origin, sigma, PT<float>::kScale), dt, px1, pa1, pxt, pat, da0, ws, wsb, st);
  if (precision == kFP64)
    return so_gradient<double, kTpb64, kRt64, kTpb64, kRt64>(
        xt, at, n, T, make_frame(origin, sigma, PT<double>::kScale), dt, px1, pa1, pxt, pat, da0, ws, wsb, st);
  return kInvalidArgument;
}

int lddmm_first_order_shoot(const double* x0, const double* at, int64_t n, int64_t T, double sigma, double regweight,
                            const double* origin, double* xt, double* energy, int precision, void* ws, size_t wsb,
                            lddmm_stream_t stream) {
  if (n < 0 || T < 0 || bad_sigma(sigma) || bad(x0, n) || bad(at, n) || bad(xt, n)) return kInvalidArgument;
  cudaStream_t st = (cudaStream_t)stream;
  const size_t stride = (size_t)n * 3;
  if (n == 0) return kOk;
  if (cudaMemcpyAsync(xt, x0, stride * sizeof(double), cudaMemcpyDeviceToDevice, st) != cudaSuccess) return kCudaError;
  if (T == 0 && energy) {
    if (cudaMemsetAsync(energy, 0, sizeof(double), st) != cudaSuccess) return kCudaError;
  }
  const double dt = T > 0 ? 1.0 / (double)T : 0.0;
  for (int64_t t = 0; t < T; ++t) {
    const double* x = xt + t * stride;
    const double* a = at + t * stride;
    int rc;
    if (precision == kFP32Compensated)
      rc = k_energy_and_update<float, kTpbLight, kRtLight>(x, a, n, make_frame(origin, sigma, PT<float>::kScale), x,
                                                           1.0, dt, xt + (t + 1) * stride, a, energy,
                                                           regweight * dt, t > 0, ws, wsb, st);
    else if (precision == kFP64)
      rc = k_energy_and_update<double, kTpb64, kRt64>(x, a, n, make_frame(origin, sigma, PT<double>::kScale), x, 1.0,
                                                      dt, xt + (t + 1) * stride, a, energy, regweight * dt, t > 0, ws,
                                                      wsb, st);
    else
      return kInvalidArgument;
    if (rc != kOk) return rc;
  }
  return kOk;
}

int lddmm_first_order_gradient(const double* xt, const double* at, int64_t n, int64_t T, double sigma,
                               double regweight, const double* px1, int euclidean, const double* origin, double* pxt,
                               double* dat, int precision, void* ws, size_t wsb, lddmm_stream_t stream) {
  if (n < 0 || T < 0 || bad_sigma(sigma) || bad(xt, n) || bad(at, n) || bad(px1, n) || bad(pxt, n) || bad(dat, n))
    return kInvalidArgument;
  if (n == 0) return kOk;
  cudaStream_t st = (cudaStream_t)stream;
  const size_t stride = (size_t)n * 3;
  if (cudaMemcpyAsync(pxt + T * stride, px1, stride * sizeof(double), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    return kCudaError;
  const double dt = T > 0 ? 1.0 / (double)T : 0.0;
  for (int64_t t = T - 1; t >= 0; --t) {
    int rc;
    if (precision == kFP32Compensated) {
      OpFOBwd<float>::Params P{xt + t * stride, at + t * stride, pxt + (t + 1) * stride, pxt + t * stride,
                               dat + t * stride, make_frame(origin, sigma, PT<float>::kScale), dt, regweight,
                               euclidean};
      rc = run_pairs<OpFOBwd<float>, float, kTpbLight, kRtLight>(P, n, n, ws, wsb, st, kCtasPerSm);
    } else if (precision == kFP64) {
      OpFOBwd<double>::Params P{xt + t * stride, at + t * stride, pxt + (t + 1) * stride, pxt + t * stride,
                                dat + t * stride, make_frame(origin, sigma, PT<double>::kScale), dt, regweight,
                                euclidean};
      rc = run_pairs<OpFOBwd<double>, double, kTpb64, kRt64>(P, n, n, ws, wsb, st, kCtasPerSm);
    } else {
      return kInvalidArgument;
    }
    if (rc != kOk) return rc;
  }
  return kOk;
}

}  // extern "C"
