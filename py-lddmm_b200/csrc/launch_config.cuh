// Launch shapes of the all-pairs kernels (threads per CTA x targets per thread), chosen for 148 SMs.
#pragma once

namespace lddmm {

// Light ops (<= 6 accumulators per target): 4 targets per thread amortise each broadcast LDS over 4 pairs.
constexpr int kTpbLight = 128;
constexpr int kRtLight = 4;
// Heavy ops (7-16 accumulators per target): 2 targets per thread keeps registers under 128.
constexpr int kTpbHeavy = 128;
constexpr int kRtHeavy = 2;
// FP64 baseline path.
constexpr int kTpb64 = 128;
constexpr int kRt64 = 2;
// Source-chunk split: aim for this many resident CTAs per SM when the target blocks alone are too few.
constexpr int kCtasPerSm = 4;

}  // namespace lddmm
