// Mixed-precision pair records: FP64 position and velocity (differences are
// formed in FP64), FP32 for everything else.
#pragma once

namespace sphgpu {

constexpr int MRECW = 14;    // SPH, in doubles: 6 FP64 + 16 FP32 slots (112 bytes)
constexpr int CMRECW = 20;   // CRKSPH, in doubles: 6 FP64 + 28 FP32 slots (160 bytes)

}  // namespace sphgpu
