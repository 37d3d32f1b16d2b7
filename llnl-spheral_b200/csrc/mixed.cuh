// Mixed-precision pair record: FP64 position and velocity (differences are
// formed in FP64), FP32 for everything else.  112 bytes per node.
#pragma once

namespace sphgpu {

constexpr int MRECW = 14;   // in doubles: 6 FP64 + 16 FP32 slots

int prepare_mixed(Problem& p);

}  // namespace sphgpu
