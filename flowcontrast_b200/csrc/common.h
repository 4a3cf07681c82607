// Constants and plain structs shared by the host runtime and the device kernels.
#pragma once
#include <cstdint>

namespace fslbm {

constexpr int kTX = 32;                 // step tile width along x (one warp per tile row)
constexpr int kTY = 8;                  // step tile height along y
constexpr int kThreads = kTX * kTY;
constexpr uint8_t kWall = 125;          // mask value of a wall cell (pipe.m:45-47)
constexpr uint8_t kGhost = 2;           // periodic image cell of a cross-section periodic in x, y

// Per cross-section column: static wall sums of the predictor and the fluid flag.
template <class TC> struct ColCoef {
  TC ws0, wsx, wsy, fluid;
};

// Per cell, for masks that vary along z: wall sums of the predictor over the 3x3x3
// neighbourhood, including the streamwise moment (zero for extruded masks).
template <class TC> struct CellCoef {
  TC ws0, wsx, wsy, wsz;
};

}  // namespace fslbm
