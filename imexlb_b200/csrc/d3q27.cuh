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
#define IMX_HDC __host__ __device__ constexpr
#else
#define IMX_HD inline
#define IMX_HDC constexpr
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
IMX_HDC double weight_of_class(int c) {
  return c == 0 ? 8.0 / 27.0 : (c == 1 ? 2.0 / 27.0 : (c == 2 ? 1.0 / 54.0 : 1.0 / 216.0));
}

// Wall record of one row (j, k) of a 2-byte standard cavity: 32 values of
// 16 bits.  Slot m of the lo side, values [0, 16), holds the post-collision
// population P_m + 1 (e_x = -1) of the cell (0, j, k); slot m of the hi side,
// values [16, 32), the population P_m (e_x = +1) of the cell (nx - 1, j, k);
// P_m is the m-th population with e_x = +1.  Those are the values that the
// halfway bounce-back at the x walls returns to the same cells one step
// later.  Slots 9-15 of a side are zero.
struct WallRecord {
  static constexpr int WORDS = 32;  // 16-bit values per row
  static constexpr int HI = 16;     // first value of the hi side
  static constexpr int BYTES = 64;
  static constexpr int SLOTS = 9;
  // P_m: 1, 7, 9, 11, 13, 19, 21, 23, 25
  static constexpr int pos(int m) { return m == 0 ? 1 : (m <= 4 ? 7 + 2 * (m - 1) : 19 + 2 * (m - 5)); }
  // slot of population q (e_x != 0): the index of P_m = q or q - 1
  static constexpr int slot(int q) {
    const int p = (q & 1) ? q : q - 1;
    return p == 1 ? 0 : (p <= 13 ? (p - 7) / 2 + 1 : (p - 19) / 2 + 5);
  }
};

constexpr bool wall_record_matches() {
  for (int m = 0; m < WallRecord::SLOTS; ++m) {
    const int p = WallRecord::pos(m);
    if (D3Q27::ex[p] != 1 || D3Q27::bb[p] != p + 1 || WallRecord::slot(p) != m || WallRecord::slot(p + 1) != m)
      return false;
  }
  return true;
}
static_assert(wall_record_matches(), "wall record slots follow the e_x = +1 populations");

}  // namespace imx
