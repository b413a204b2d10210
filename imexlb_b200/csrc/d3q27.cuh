// D3Q27 lattice constants and the arithmetic building blocks of the fused
// step, shared by host and device code.
//
// The velocity set, weights and opposite-direction table use the reference's
// ordering (tgv/src/lbm.cpp:27-190): 0 rest; 1-6 the axes +x,-x,+y,-y,+z,-z;
// 7-18 the twelve edge directions; 19-26 the eight corners.  Opposite pairs
// are adjacent (q, q+1) for q odd.
#pragma once

#include <cstdint>

#if defined(__CUDACC__)
#define IMX_HD __host__ __device__ __forceinline__
#else
#define IMX_HD inline
#endif

namespace imx {

constexpr int Q = 27;
constexpr int GHOST = 3;  // ghost width of the reference layout (tgv/src/lbm.hpp:22)

struct D3Q27 {
  static constexpr int ex[Q] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1};
  static constexpr int ey[Q] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1, -1, 1};
  static constexpr int ez[Q] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1, -1, 1, -1, 1};
  static constexpr int bb[Q] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17, 20, 19, 22, 21, 24, 23, 26, 25};
  // weight class: 0 rest (8/27), 1 axis (2/27), 2 edge (1/54), 3 corner (1/216)
  static constexpr int wclass[Q] = {0, 1, 1, 1, 1, 1, 1, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 3, 3, 3, 3, 3, 3, 3, 3};
};

// The weights as the reference computes them: 8.0/27.0, 2.0/27.0, 1.0/54.0,
// 1.0/216.0 (each a correctly rounded double quotient).
IMX_HD double weight_of_class(int c) {
  return c == 0 ? 8.0 / 27.0 : (c == 1 ? 2.0 / 27.0 : (c == 2 ? 1.0 / 54.0 : 1.0 / 216.0));
}

}  // namespace imx
