// lddmm_apply_k_static: the Gaussian kernel sum K(y, x) a without a caller-provided workspace.
//
// Who needs it: callers that cannot allocate device memory when they call us. A host application that fixes its
// whole device-memory budget at start-up, or a plugin host that owns the device memory and hands its plugins no
// allocator, has nowhere to get the workspace that lddmm_apply_k needs; and code on a latency-critical path may not
// call cudaMalloc at all, because the call can synchronise the whole device. This entry point takes only inputs and
// outputs and never allocates: its scratch (the stream-K partial sums) lives in a fixed array compiled into this
// library, which every GPU that loads the library holds (32 MiB) until the process exits.
//
// Limits and rules (repeated in include/lddmm_b200.h):
//  - at most kStaticMaxTargets = 262,144 targets. The scratch of K a is its stream-K partial sums alone (the sum is
//    not culled, so no coordinate boxes are kept): at most (C / gx + 2) slots of 3 partials per target, C resident
//    CTAs and gx target blocks, whatever the number of sources. On a B200 (148 SMs; 3 CTAs per SM for the FP32
//    kernel, 1,024 targets per block) the largest such request needs 20.7 MiB (n = 226,301: 4 slots), so every
//    request with at most 262,144 targets fits the 32 MiB array for any source count up to the library's limit of
//    536,870,911. A request that would not fit (a device with many more resident CTAs) is rejected before any
//    launch with LDDMM_ERR_WORKSPACE;
//  - the first call on a device looks up the array's device address (cudaGetSymbolAddress) with that device
//    current; make that first call before any stream capture on the device;
//  - every call shares the one array and leaves its partial sums in it. Nothing needs clearing between calls: each
//    call writes every slot it later reads. Calls that overlap on the GPU (two streams, or two host threads) race
//    on the array and give wrong results: serialise them.
#include <mutex>

#include "../../include/lddmm_b200.h"
#include "kernel_ops.cuh"
#include "launch_config.cuh"

namespace lddmm {
namespace {

constexpr size_t kStaticScratchBytes = size_t(32) << 20;
constexpr int64_t kStaticMaxTargets = 262144;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_apply_k_scratch[kStaticScratchBytes];

std::mutex g_scratch_mutex;
void* g_scratch_address[kMaxDevices] = {};

// Device address of the scratch array on the current device, looked up once per device.
int scratch_on_current_device(void** address) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return kCudaError;
  }
  if (dev < 0 || dev >= kMaxDevices) return kUnsupported;
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (g_scratch_address[dev] == nullptr) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_apply_k_scratch) != cudaSuccess || p == nullptr) {
      cudaGetLastError();
      return kCudaError;
    }
    g_scratch_address[dev] = p;
  }
  *address = g_scratch_address[dev];
  return kOk;
}

bool missing(const void* p, int64_t count) { return count > 0 && p == nullptr; }

}  // namespace
}  // namespace lddmm

using namespace lddmm;

extern "C" int lddmm_apply_k_static(const double* y, int64_t n, const double* x, const double* a, int64_t m,
                                    double sigma, const double* origin, double* out, int precision,
                                    lddmm_stream_t stream) {
  if (n < 0 || m < 0 || bad_sigma(sigma) || missing(y, n) || missing(out, n) || missing(x, m) || missing(a, m))
    return kInvalidArgument;
  if (precision != kFP32Compensated && precision != kFP64) return kInvalidArgument;
  if (n > kStaticMaxTargets) return kWorkspaceTooSmall;
  if (n == 0) return kOk;
  void* scratch = nullptr;
  const int rc = scratch_on_current_device(&scratch);
  if (rc != kOk) return rc;
  OpK::Params P;
  P.y = y;
  P.x = x;
  P.a = a;
  P.out = out;
  cudaStream_t st = (cudaStream_t)stream;
  if (precision == kFP32Compensated) {
    P.f = make_frame(origin, sigma, kGauss, true);
    return run_pairs<OpK, F2, kTpbLight, kRtLight>(P, n, m, scratch, kStaticScratchBytes, st);
  }
  P.f = make_frame(origin, sigma, kGauss, false);
  return run_pairs<OpK, double, kTpb64, kRt64>(P, n, m, scratch, kStaticScratchBytes, st);
}
