// C-ABI entry points of the kernel operators (Kernel.applyK / applyDiffKT / applyDDiffK11and12 /
// applyDiffK1and2 / applyDivergence / applyKTensor).
#include "../../include/lddmm_b200.h"
#include "kernel_ops.cuh"
#include "launch_config.cuh"
#include "pairs_sym.cuh"

namespace lddmm {

int device_sm_count() {
  static int cached = 0;
  if (cached > 0) return cached;
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) {
    cudaGetLastError();
    return 148;
  }
  cached = sms;
  return sms;
}

int resident_ctas(const void* kernel, int threads, size_t dynamic_smem) {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, dynamic_smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
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

template <class Op, int TPB32, int RT32, class Fill>
int dispatch(int precision, int64_t n, int64_t m, double sigma, int kernel, const double* origin, void* ws,
             size_t wsb, cudaStream_t st, Fill fill) {
  if (bad_kernel(kernel)) return kInvalidArgument;
  typename Op::Params P;
  if (precision == kFP32Compensated) {
    P.f = make_frame(origin, sigma, kernel, true);
    fill(P);
    return run_pairs_k<Op, F2, TPB32, RT32>(P, n, m, ws, wsb, st);
  } else if (precision == kFP64) {
    P.f = make_frame(origin, sigma, kernel, false);
    fill(P);
    return run_pairs_k<Op, double, kTpb64, kRt64>(P, n, m, ws, wsb, st);
  }
  return kInvalidArgument;
}

template <class Op, int TPB32, int RT32>
size_t op_ws(int64_t n, int64_t m, int precision) {
  return precision == kFP32Compensated ? pairs_ws_bytes_any<Op, F2, TPB32, RT32>(n, m)
                                       : pairs_ws_bytes_any<Op, double, kTpb64, kRt64>(n, m);
}

}  // namespace

size_t kernel_sums_ws_bytes(int64_t n, int64_t m, int precision) {
  size_t b = 0;
  auto upd = [&](size_t v) { b = v > b ? v : b; };
  upd(op_ws<OpK, kTpbLight, kRtLight>(n, m, precision));
  upd(op_ws<OpDiffKT<0>, kTpbLight, kRtLight>(n, m, precision));
  upd(op_ws<OpDiffKT<1>, kTpbLight, kRtLight>(n, m, precision));
  upd(op_ws<OpDiffKT<2>, kTpbLight, kRtLight>(n, m, precision));
  upd(op_ws<OpDDiffK, kTpbHeavy, kRtHeavy>(n, m, precision));
  upd(op_ws<OpDiffK1and2, kTpbLight, kRtLight>(n, m, precision));
  upd(op_ws<OpDiv, kTpbLight, kRtLight>(n, m, precision));
  upd(op_ws<OpKTensor, kTpbLight, kRtLight>(n, m, precision));
  if (LDDMM_SYM && precision == kFP32Compensated && n == m) {
    upd(symx_ws_bytes<OpKSym, kTpbKSym, kRtKSym>(n));
    upd(sym_ws_bytes<OpKSymD, kTpbLight, kRtKSymL, Laplacian>(n));
  }
  return b;
}

}  // namespace lddmm

using namespace lddmm;

extern "C" {

int lddmm_apply_k(const double* y, int64_t n, const double* x, const double* a, int64_t m, double sigma, int kernel,
                  const double* origin, double* out, int precision, void* ws, size_t wsb, lddmm_stream_t stream) {
  if (n < 0 || m < 0 || bad_sigma(sigma) || bad_ptr(y, n) || bad_ptr(out, n) || bad_ptr(x, m) || bad_ptr(a, m))
    return kInvalidArgument;
  // a self-sum K(x, x) a (the same point array as targets and sources): each unordered pair once
  if (LDDMM_SYM && precision == kFP32Compensated && y == x && n == m && !bad_kernel(kernel)) {
    OpK::Params P;
    P.f = make_frame(origin, sigma, kernel, true);
    P.y = y; P.x = x; P.a = a; P.out = out;
    if (kernel == kGauss) return run_pairs_symx<OpKSym, kTpbKSym, kRtKSym>(P, n, ws, wsb, (cudaStream_t)stream);
    return run_pairs_sym<OpKSymD, kTpbLight, kRtKSymL, Laplacian>(P, n, ws, wsb, (cudaStream_t)stream);
  }
  return dispatch<OpK, kTpbLight, kRtLight>(precision, n, m, sigma, kernel, origin, ws, wsb, (cudaStream_t)stream,
                                            [&](OpK::Params& P) { P.y = y; P.x = x; P.a = a; P.out = out; });
}

int lddmm_apply_diff_kt(const double* y, int64_t n, const double* x, const double* p, const double* a, int64_t m,
                        double sigma, int kernel, int mode, double regweight, const double* origin, double* out,
                        int precision, void* ws, size_t wsb, lddmm_stream_t stream) {
  if (n < 0 || m < 0 || bad_sigma(sigma) || bad_ptr(y, n) || bad_ptr(out, n) || bad_ptr(p, n) || bad_ptr(x, m) ||
      bad_ptr(a, m) || mode < 0 || mode > 2)
    return kInvalidArgument;
  if (mode != 0 && n != m) return kInvalidArgument;
  auto fill = [&](auto& P) { P.y = y; P.x = x; P.p = p; P.a = a; P.out = out; P.w = regweight; };
  cudaStream_t st = (cudaStream_t)stream;
  if (mode == 0)
    return dispatch<OpDiffKT<0>, kTpbLight, kRtLight>(precision, n, m, sigma, kernel, origin, ws, wsb, st, fill);
  if (mode == 1)
    return dispatch<OpDiffKT<1>, kTpbLight, kRtLight>(precision, n, m, sigma, kernel, origin, ws, wsb, st, fill);
  return dispatch<OpDiffKT<2>, kTpbLight, kRtLight>(precision, n, m, sigma, kernel, origin, ws, wsb, st, fill);
}

int lddmm_apply_ddiff_k11and12(const double* x, const double* nn, const double* a, const double* p, int64_t n,
                               double sigma, int kernel, const double* origin, double* out, int precision, void* ws,
                               size_t wsb, lddmm_stream_t stream) {
  if (n < 0 || bad_sigma(sigma) || bad_ptr(x, n) || bad_ptr(nn, n) || bad_ptr(a, n) || bad_ptr(p, n) ||
      bad_ptr(out, n))
    return kInvalidArgument;
  auto fill = [&](OpDDiffK::Params& P) { P.x = x; P.nn = nn; P.a = a; P.p = p; P.out = out; };
  return dispatch<OpDDiffK, kTpbHeavy, kRtHeavy>(precision, n, n, sigma, kernel, origin, ws, wsb,
                                                 (cudaStream_t)stream, fill);
}

int lddmm_apply_diff_k1and2(const double* x, const double* a1, const double* a2, int64_t n, double sigma, int kernel,
                            const double* origin, double* out, int precision, void* ws, size_t wsb,
                            lddmm_stream_t stream) {
  if (n < 0 || bad_sigma(sigma) || bad_ptr(x, n) || bad_ptr(a1, n) || bad_ptr(a2, n) || bad_ptr(out, n))
    return kInvalidArgument;
  auto fill = [&](OpDiffK1and2::Params& P) { P.x = x; P.a1 = a1; P.a2 = a2; P.out = out; };
  return dispatch<OpDiffK1and2, kTpbLight, kRtLight>(precision, n, n, sigma, kernel, origin, ws, wsb,
                                                     (cudaStream_t)stream, fill);
}

int lddmm_apply_divergence(const double* y, int64_t n, const double* x, const double* a, int64_t m, double sigma,
                           int kernel, const double* origin, double* out, int precision, void* ws, size_t wsb,
                           lddmm_stream_t stream) {
  if (n < 0 || m < 0 || bad_sigma(sigma) || bad_ptr(y, n) || bad_ptr(out, n) || bad_ptr(x, m) || bad_ptr(a, m))
    return kInvalidArgument;
  return dispatch<OpDiv, kTpbLight, kRtLight>(precision, n, m, sigma, kernel, origin, ws, wsb, (cudaStream_t)stream,
                                              [&](OpDiv::Params& P) { P.y = y; P.x = x; P.a = a; P.out = out; });
}

int lddmm_apply_k_tensor(const double* y, int64_t n, const double* x, int64_t m, const double* ay, const double* ax,
                         const double* by, const double* bx, double sigma, const double* origin, double* out,
                         int precision, void* ws, size_t wsb, lddmm_stream_t stream) {
  if (n < 0 || m < 0 || bad_sigma(sigma) || bad_ptr(y, n) || bad_ptr(ay, n) || bad_ptr(by, n) || bad_ptr(out, n) ||
      bad_ptr(x, m) || bad_ptr(ax, m) || bad_ptr(bx, m))
    return kInvalidArgument;
  auto fill = [&](OpKTensor::Params& P) {
    P.y = y; P.x = x; P.ay = ay; P.ax = ax; P.by = by; P.bx = bx; P.out = out;
  };
  return dispatch<OpKTensor, kTpbLight, kRtLight>(precision, n, m, sigma, kGauss, origin, ws, wsb,
                                                  (cudaStream_t)stream, fill);
}

}  // extern "C"
