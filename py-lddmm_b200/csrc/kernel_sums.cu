// C-ABI entry points of the Gaussian kernel operators (Kernel.applyK / applyDiffKT / applyDDiffK11and12 /
// applyDiffK1and2 / applyDivergence / applyKTensor and the dense-weight variants).
#include "../../include/lddmm_b200.h"
#include "kernel_ops.cuh"
#include "launch_config.cuh"

namespace lddmm {

int device_sm_count() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) return 148;
  return sms;
}

__global__ void ordered_sum_kernel(const double* __restrict__ v, int count, double scale, double* out,
                                   int accumulate) {
  __shared__ double red[1024];
  double s = 0.0;
  for (int i = threadIdx.x; i < count; i += blockDim.x) s += v[i];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = (accumulate ? out[0] : 0.0) + scale * red[0];
}

namespace {

bool bad_ptr(const void* p, int64_t count) { return count > 0 && p == nullptr; }

template <template <typename> class OpT, int TPB32, int RT32, int TPB64, int RT64, class Fill>
int dispatch(int precision, int64_t n, int64_t m, double sigma, const double* origin, void* ws, size_t wsb,
             cudaStream_t st, Fill fill) {
  if (precision == kFP32Compensated) {
    typename OpT<float>::Params P;
    P.f = make_frame(origin, sigma, PT<float>::kScale);
    fill(P);
    return run_pairs<OpT<float>, float, TPB32, RT32>(P, n, m, ws, wsb, st, kCtasPerSm);
  } else if (precision == kFP64) {
    typename OpT<double>::Params P;
    P.f = make_frame(origin, sigma, PT<double>::kScale);
    fill(P);
    return run_pairs<OpT<double>, double, TPB64, RT64>(P, n, m, ws, wsb, st, kCtasPerSm);
  }
  return kInvalidArgument;
}

template <typename R> using OpDiffKT0 = OpDiffKT<R, 0>;
template <typename R> using OpDiffKT1 = OpDiffKT<R, 1>;
template <typename R> using OpDiffKT2 = OpDiffKT<R, 2>;

}  // namespace

size_t kernel_sums_ws_bytes(int64_t n, int64_t m, int precision) {
  size_t b = 0;
  auto upd = [&](size_t v) { b = v > b ? v : b; };
  if (precision == kFP32Compensated) {
    upd(pairs_ws_bytes<OpK<float>, float, kTpbLight, kRtLight>(n, m, kCtasPerSm));
    upd(pairs_ws_bytes<OpDiffKT<float, 2>, float, kTpbLight, kRtLight>(n, m, kCtasPerSm));
    upd(pairs_ws_bytes<OpDDiffK<float>, float, kTpbHeavy, kRtHeavy>(n, m, kCtasPerSm));
    upd(pairs_ws_bytes<OpDiffK1and2<float>, float, kTpbLight, kRtLight>(n, m, kCtasPerSm));
    upd(pairs_ws_bytes<OpKTensor<float>, float, kTpbLight, kRtLight>(n, m, kCtasPerSm));
  } else {
    upd(pairs_ws_bytes<OpK<double>, double, kTpb64, kRt64>(n, m, kCtasPerSm));
    upd(pairs_ws_bytes<OpDDiffK<double>, double, kTpb64, kRt64>(n, m, kCtasPerSm));
  }
  return b;
}

}  // namespace lddmm

using namespace lddmm;

extern "C" {

int lddmm_apply_k(const double* y, int64_t n, const double* x, const double* a, int64_t m, double sigma,
                  const double* origin, double* out, int precision, void* ws, size_t wsb, lddmm_stream_t stream) {
  if (n < 0 || m < 0 || bad_sigma(sigma) || bad_ptr(y, n) || bad_ptr(out, n) || bad_ptr(x, m) || bad_ptr(a, m))
    return kInvalidArgument;
  return dispatch<OpK, kTpbLight, kRtLight, kTpb64, kRt64>(precision, n, m, sigma, origin, ws, wsb,
                                                             (cudaStream_t)stream, [&](auto& P) {
    P.y = y; P.x = x; P.a = a; P.out = out;
  });
}

int lddmm_apply_diff_kt(const double* y, int64_t n, const double* x, const double* p, const double* a, int64_t m,
                        double sigma, int mode, double regweight, const double* origin, double* out, int precision,
                        void* ws, size_t wsb, lddmm_stream_t stream) {
  if (n < 0 || m < 0 || bad_sigma(sigma) || bad_ptr(y, n) || bad_ptr(out, n) || bad_ptr(p, n) || bad_ptr(x, m) ||
      bad_ptr(a, m) || mode < 0 || mode > 2)
    return kInvalidArgument;
  if (mode != 0 && n != m) return kInvalidArgument;
  auto fill = [&](auto& P) { P.y = y; P.x = x; P.p = p; P.a = a; P.out = out; P.w = regweight; };
  cudaStream_t st = (cudaStream_t)stream;
  if (mode == 0) return dispatch<OpDiffKT0, kTpbLight, kRtLight, kTpb64, kRt64>(precision, n, m, sigma, origin, ws, wsb, st, fill);
  if (mode == 1) return dispatch<OpDiffKT1, kTpbLight, kRtLight, kTpb64, kRt64>(precision, n, m, sigma, origin, ws, wsb, st, fill);
  return dispatch<OpDiffKT2, kTpbLight, kRtLight, kTpb64, kRt64>(precision, n, m, sigma, origin, ws, wsb, st, fill);
}

int lddmm_apply_ddiff_k11and12(const double* x, const double* nn, const double* a, const double* p, int64_t n,
                               double sigma, const double* origin, double* out, int precision, void* ws,
                               size_t wsb, lddmm_stream_t stream) {
  if (n < 0 || bad_sigma(sigma) || bad_ptr(x, n) || bad_ptr(nn, n) || bad_ptr(a, n) || bad_ptr(p, n) ||
      bad_ptr(out, n))
    return kInvalidArgument;
  return dispatch<OpDDiffK, kTpbHeavy, kRtHeavy, kTpb64, kRt64>(precision, n, n, sigma, origin, ws, wsb,
                                                                  (cudaStream_t)stream, [&](auto& P) {
    P.x = x; P.nn = nn; P.a = a; P.p = p; P.out = out;
  });
}

int lddmm_apply_diff_k1and2(const double* x, const double* a1, const double* a2, int64_t n, double sigma,
                            const double* origin, double* out, int precision, void* ws, size_t wsb,
                            lddmm_stream_t stream) {
  if (n < 0 || bad_sigma(sigma) || bad_ptr(x, n) || bad_ptr(a1, n) || bad_ptr(a2, n) || bad_ptr(out, n))
    return kInvalidArgument;
  return dispatch<OpDiffK1and2, kTpbLight, kRtLight, kTpb64, kRt64>(precision, n, n, sigma, origin, ws, wsb,
                                                                      (cudaStream_t)stream, [&](auto& P) {
    P.x = x; P.a1 = a1; P.a2 = a2; P.out = out;
  });
}

int lddmm_apply_divergence(const double* y, int64_t n, const double* x, const double* a, int64_t m, double sigma,
                           const double* origin, double* out, int precision, void* ws, size_t wsb,
                           lddmm_stream_t stream) {
  if (n < 0 || m < 0 || bad_sigma(sigma) || bad_ptr(y, n) || bad_ptr(out, n) || bad_ptr(x, m) || bad_ptr(a, m))
    return kInvalidArgument;
  return dispatch<OpDiv, kTpbLight, kRtLight, kTpb64, kRt64>(precision, n, m, sigma, origin, ws, wsb,
                                                               (cudaStream_t)stream, [&](auto& P) {
    P.y = y; P.x = x; P.a = a; P.out = out;
  });
}

int lddmm_apply_k_tensor(const double* y, int64_t n, const double* x, int64_t m, const double* ay, const double* ax,
                         const double* by, const double* bx, double sigma, const double* origin, double* out,
                         int precision, void* ws, size_t wsb, lddmm_stream_t stream) {
  if (n < 0 || m < 0 || bad_sigma(sigma) || bad_ptr(y, n) || bad_ptr(ay, n) || bad_ptr(by, n) || bad_ptr(out, n) ||
      bad_ptr(x, m) || bad_ptr(ax, m) || bad_ptr(bx, m))
    return kInvalidArgument;
  return dispatch<OpKTensor, kTpbLight, kRtLight, kTpb64, kRt64>(precision, n, m, sigma, origin, ws, wsb,
                                                                   (cudaStream_t)stream, [&](auto& P) {
    P.y = y; P.x = x; P.ay = ay; P.ax = ax; P.by = by; P.bx = bx; P.out = out;
  });
}

}  // extern "C"
