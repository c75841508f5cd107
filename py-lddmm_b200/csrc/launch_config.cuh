// Launch shapes of the all-pairs kernels (threads per CTA x targets per thread). The defaults were chosen by
// timing on the B200; each can be overridden at build time (-DLDDMM_RT_LIGHT=... etc.) for tuning sweeps.
#pragma once
#include <stdint.h>

#ifndef LDDMM_TPB_LIGHT
#define LDDMM_TPB_LIGHT 128
#endif
#ifndef LDDMM_RT_LIGHT
#define LDDMM_RT_LIGHT 4
#endif
#ifndef LDDMM_TPB_HEAVY
#define LDDMM_TPB_HEAVY 128
#endif
#ifndef LDDMM_RT_HEAVY
#define LDDMM_RT_HEAVY 2
#endif
#ifndef LDDMM_RT_ADJOINT
#define LDDMM_RT_ADJOINT 4
#endif
#ifndef LDDMM_RT_SYM_FWD
#define LDDMM_RT_SYM_FWD 8
#endif
#ifndef LDDMM_RT_FO_SYM
#define LDDMM_RT_FO_SYM 4
#endif
#ifndef LDDMM_RT_SYM_SMALL
#define LDDMM_RT_SYM_SMALL 2
#endif
#ifndef LDDMM_SYM_FWD_SMALL_N
#define LDDMM_SYM_FWD_SMALL_N 16384
#endif
#ifndef LDDMM_SYM_ADJ_SMALL_N
#define LDDMM_SYM_ADJ_SMALL_N 6144
#endif
#ifndef LDDMM_RT_SYM_FWD_L
#define LDDMM_RT_SYM_FWD_L 4
#endif
#ifndef LDDMM_RT_ADJOINT_SYM_L
#define LDDMM_RT_ADJOINT_SYM_L 2
#endif
#ifndef LDDMM_RT_FO_SYM_L
#define LDDMM_RT_FO_SYM_L 4
#endif
#ifndef LDDMM_RT_KSYM_L
#define LDDMM_RT_KSYM_L 4
#endif
#ifndef LDDMM_TPB_KSYM
#define LDDMM_TPB_KSYM 128
#endif
#ifndef LDDMM_RT_KSYM
#define LDDMM_RT_KSYM 8
#endif
#ifndef LDDMM_TPB_64
#define LDDMM_TPB_64 128
#endif
#ifndef LDDMM_RT_64
#define LDDMM_RT_64 2
#endif

namespace lddmm {

// Light ops (<= 8 accumulators per target): several targets per thread amortise each broadcast LDS.
constexpr int kTpbLight = LDDMM_TPB_LIGHT;
constexpr int kRtLight = LDDMM_RT_LIGHT;
// Heavy ops (the 7-accumulator DDK): fewer targets per thread.
constexpr int kTpbHeavy = LDDMM_TPB_HEAVY;
constexpr int kRtHeavy = LDDMM_RT_HEAVY;
// The 12-accumulator second-order adjoint step: 4 targets per thread with its sums in registers (254 registers,
// 2 CTAs per SM) measured 4% faster than 2 targets per thread at 4 CTAs per SM (half the shared-memory reads per
// pair, two independent lane groups per source).
constexpr int kRtAdjoint = LDDMM_RT_ADJOINT;
// The symmetric second-order forward step (pairs_kernel_sym): 8 targets per thread (168 registers, 3 CTAs per SM,
// its compensated row sums in 48 KiB of dynamic shared memory) measured 15% faster at level 6 than 4 targets per
// thread (134 registers, 3 CTAs per SM): the per-step source loads and the column shuffles are shared by twice
// as many pairs, and four independent lane groups hide the latency of the ex2 chain.
constexpr int kRtSymFwd = LDDMM_RT_SYM_FWD;
// Small point sets (the coarse levels of a coarse-to-fine registration): row blocks of 256 points instead of 1,024
// (forward) or 512 (adjoint), so that the unit triangle gives the GPU ~10x more units. At level 4 (2,562 points)
// 1,024-point blocks leave 39 units for 444 resident CTAs and a step is latency-bound (39.5 us forward, 39.4 us
// adjoint, with the epilogue); 2 targets per thread: 27.2 and 31.2 us. At level 5 (10,242) the forward step
// still gains (123.5 -> 95.7 us) and the adjoint step loses (134.4 -> 146.6 us); at level 6 both lose 30-40%.
constexpr int kRtSymSmall = LDDMM_RT_SYM_SMALL;
constexpr int64_t kSymFwdSmallN = LDDMM_SYM_FWD_SMALL_N;  // Gaussian forward step: 2 targets per thread up to here
constexpr int64_t kSymAdjSmallN = LDDMM_SYM_ADJ_SMALL_N;  // Gaussian adjoint step: 2 targets per thread up to here
// The symmetric K(x, x) a (pairs_kernel_symx): 8 targets per thread.
// The symmetric first-order adjoint step (pairs_kernel_sym): 4 targets per thread.
constexpr int kRtFoSym = LDDMM_RT_FO_SYM;
// The symmetric steps with the Laplacian family (its radial profile -- a square root and the polynomial -- takes
// registers that the Gaussian shapes spend on more targets per thread).
constexpr int kRtSymFwdL = LDDMM_RT_SYM_FWD_L;
constexpr int kRtAdjointSymL = LDDMM_RT_ADJOINT_SYM_L;
constexpr int kRtFoSymL = LDDMM_RT_FO_SYM_L;
constexpr int kRtKSymL = LDDMM_RT_KSYM_L;
constexpr int kTpbKSym = LDDMM_TPB_KSYM;
constexpr int kRtKSym = LDDMM_RT_KSYM;
// FP64 baseline path.
constexpr int kTpb64 = LDDMM_TPB_64;
constexpr int kRt64 = LDDMM_RT_64;

}  // namespace lddmm
