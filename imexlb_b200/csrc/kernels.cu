// Device kernels of the fused D3Q27 step (sm_100a).
//
// One kernel per time step does what the reference spreads over Collision,
// pack/exchange/unpack, Streaming and Update (tgv/main.cpp:70-134):
//
//   pull   f_q(x) = f*_q(x - e_q)             (tgv/src/lbm.cpp:243-246)
//   moments p = sum f_q / 3, u = sum f_q e_q  (tgv/src/lbm.cpp:288-333,
//                                              lid_driven_cavity/src/lbm.cpp:319-349)
//   case rules on the moments                 (cavity lid, sphere mask/inlet/outlet)
//   collide f*_q = f_q - (f_q - feq_q)/(tau0 + 0.5)   (tgv/src/lbm.cpp:222-237)
//
// so the buffer a step writes holds the post-collision distributions of the
// next step, and its moments are exactly the reference's ua, va, wa, p after
// that step.  The stencil is HBM-bound: 27 loads + 27 stores per cell, one
// thread per cell, x along threadIdx.x so each population moves as fully
// coalesced 128-byte lines.  No shared memory is needed: every value a
// thread pulls is read by exactly one thread, and the one-element x shifts of
// the 18 populations with e_x != 0 are served from L1/L2.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <type_traits>
#include <utility>

#include "lattice.h"

namespace imx {
namespace {

constexpr int RED_THREADS_DRAG = 256;

template <int A, int B, class F>
__device__ __forceinline__ void static_for(F&& f) {
  if constexpr (A < B) {
    f(std::integral_constant<int, A>{});
    static_for<A + 1, B>(f);
  }
}

// ------------------------------------------------------------ arithmetic
// EXACT: one rounding per operation in the reference's order (the __d*_rn
// intrinsics are never contracted into fused multiply-adds), and true IEEE
// division.  FAST: ordinary operators; nvcc fuses multiply-adds.
template <class R, bool EXACT> struct Ar {
  static __device__ __forceinline__ R add(R a, R b) { return a + b; }
  static __device__ __forceinline__ R sub(R a, R b) { return a - b; }
  static __device__ __forceinline__ R mul(R a, R b) { return a * b; }
};
template <> struct Ar<double, true> {
  static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
  static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
};

// e_q . (u, v, w) for e components in {-1, 0, 1}.  The reference forms
// (e0*u + e1*v) + e2*w; multiplying by +-1 is exact and adding a zero product
// leaves the sum unchanged, so dropping zero terms and negating for -1 gives
// the same value (up to the sign of an all-zero result, which no later
// operation can observe).
template <int q, class R, bool EXACT>
__device__ __forceinline__ R edu_of(R u, R v, R w) {
  using A = Ar<R, EXACT>;
  constexpr int a = D3Q27::ex[q], b = D3Q27::ey[q], c = D3Q27::ez[q];
  R t = R(0);
  if constexpr (a != 0) t = a > 0 ? u : -u;
  if constexpr (b != 0) {
    if constexpr (a != 0)
      t = b > 0 ? A::add(t, v) : A::sub(t, v);
    else
      t = b > 0 ? v : -v;
  }
  if constexpr (c != 0) {
    if constexpr (a != 0 || b != 0)
      t = c > 0 ? A::add(t, w) : A::sub(t, w);
    else
      t = c > 0 ? w : -w;
  }
  return t;
}

// RN(x / 3) in three FP64 operations (Markstein's correction step: P.
// Markstein, IBM J. Res. Dev. 34(1), 1990).  With z = RN(1/3):
//   q0 = RN(x z) is within 1.75 ulp of x/3, so r = x - 3 q0 is a multiple of
//   ulp(q0) of magnitude <= 5.25 ulp(q0): the fma computes it exactly;
//   q1 = RN(q0 + r z) = RN(x/3 + eta) with |eta| < 2^-52 ulp.
// x/3 is never within ulp/6 of a midpoint between doubles (a midpoint has an
// odd 54-bit significand, 3 times it cannot equal the 53-bit x), so q1 is
// exactly the correctly rounded quotient, as IEEE division gives.  Valid for
// zero and every x whose quotient is normal (the lattice values are O(1)).
__device__ __forceinline__ double div3_rn(double x) {
  const double z = 0x1.5555555555555p-2;
  const double q0 = __dmul_rn(x, z);
  const double r = __fma_rn(-q0, 3.0, x);
  return __fma_rn(r, z, q0);
}

template <class R>
__device__ __forceinline__ R wgt(int cls) {
  return cls == 0 ? R(8.0 / 27.0) : (cls == 1 ? R(2.0 / 27.0) : (cls == 2 ? R(1.0 / 54.0) : R(1.0 / 216.0)));
}

// Moments of the pulled populations.  EXACT follows the reference sums term
// by term in population order from a zero accumulator: p += f/3.0,
// u += f*e_x, ...  (a product with e = 0 adds nothing).
template <class R, bool EXACT>
__device__ __forceinline__ void moments(const R (&f)[Q], R& u, R& v, R& w, R& p) {
  if constexpr (EXACT) {
    using A = Ar<double, true>;
    double pm = 0.0, um = 0.0, vm = 0.0, wm = 0.0;
    static_for<0, Q>([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      pm = A::add(pm, div3_rn(f[q]));
      if constexpr (D3Q27::ex[q] == 1) um = A::add(um, f[q]);
      if constexpr (D3Q27::ex[q] == -1) um = A::sub(um, f[q]);
      if constexpr (D3Q27::ey[q] == 1) vm = A::add(vm, f[q]);
      if constexpr (D3Q27::ey[q] == -1) vm = A::sub(vm, f[q]);
      if constexpr (D3Q27::ez[q] == 1) wm = A::add(wm, f[q]);
      if constexpr (D3Q27::ez[q] == -1) wm = A::sub(wm, f[q]);
    });
    u = um;
    v = vm;
    w = wm;
    p = pm;
  } else {
    R s = R(0), um = R(0), vm = R(0), wm = R(0);
    static_for<0, Q>([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      s += f[q];
      if constexpr (D3Q27::ex[q] == 1) um += f[q];
      if constexpr (D3Q27::ex[q] == -1) um -= f[q];
      if constexpr (D3Q27::ey[q] == 1) vm += f[q];
      if constexpr (D3Q27::ey[q] == -1) vm -= f[q];
      if constexpr (D3Q27::ez[q] == 1) wm += f[q];
      if constexpr (D3Q27::ez[q] == -1) wm -= f[q];
    });
    u = um;
    v = vm;
    w = wm;
    p = s * R(1.0 / 3.0);
  }
}

// Equilibrium of the reference (tgv/src/lbm.cpp:228-232):
//   feq = t*p*3 + t*(3 edu + 4.5 edu^2 - 1.5 u.u)
template <int q, class R, bool EXACT>
__device__ __forceinline__ R feq_of(R u, R v, R w, const R (&tp3)[4], R udu15) {
  using A = Ar<R, EXACT>;
  constexpr int cls = D3Q27::wclass[q];
  const R e = edu_of<q, R, EXACT>(u, v, w);
  const R br = A::sub(A::add(A::mul(R(3.0), e), A::mul(R(4.5), A::mul(e, e))), udu15);
  return A::add(tp3[cls], A::mul(wgt<R>(cls), br));
}

template <class R, bool EXACT>
__device__ __forceinline__ void feq_prep(R u, R v, R w, R p, R (&tp3)[4], R& udu15) {
  using A = Ar<R, EXACT>;
  const R udu = A::add(A::add(A::mul(u, u), A::mul(v, v)), A::mul(w, w));
  udu15 = A::mul(R(1.5), udu);
#pragma unroll
  for (int c = 0; c < 4; ++c) tp3[c] = A::mul(A::mul(wgt<R>(c), p), R(3.0));
}

// ------------------------------------------------------------ storage
template <Store S> struct StoreT;
template <> struct StoreT<Store::F64> { using T = double; using R = double; };
template <> struct StoreT<Store::F32> { using T = float; using R = float; };
template <> struct StoreT<Store::F16> { using T = __half; using R = float; };
template <> struct StoreT<Store::BF16> { using T = __nv_bfloat16; using R = float; };

// Reduced-precision storage holds the deviation d_q = f_q - 3 w_q p_shift
// (p_shift = the rest pressure) times a per-population scale.  The step works
// on deviations throughout: their moments are (u, v, w, p - p_shift) and
// feq(u, p) - 3 w_q p_shift = feq(u, p - p_shift), so nothing large cancels in
// FP32.  FP64 storage keeps f itself (p_shift = 0).
template <Store S>
__device__ __forceinline__ typename StoreT<S>::R decode(typename StoreT<S>::T x, int q, const Encoding& e) {
  if constexpr (S == Store::F64 || S == Store::F32) {
    return x;
  } else if constexpr (S == Store::F16) {
    return __half2float(x) * e.inv_scale[q];
  } else {
    return __bfloat162float(x) * e.inv_scale[q];
  }
}
template <Store S>
__device__ __forceinline__ typename StoreT<S>::T encode(typename StoreT<S>::R x, int q, const Encoding& e) {
  if constexpr (S == Store::F64 || S == Store::F32) {
    return x;
  } else if constexpr (S == Store::F16) {
    return __float2half_rn(x * e.scale[q]);
  } else {
    return __float2bfloat16_rn(x * e.scale[q]);
  }
}

template <class T>
__device__ __forceinline__ T ldg_stream(const T* p) {
  return __ldg(p);
}

// ------------------------------------------------------------ init
// f = feq(u, v, w, p) over every stored cell, into both buffers (the
// reference initialises the whole padded box, tgv/src/lbm.cpp:209-218).  The
// macroscopic fields cover the stored box (x fastest).
template <Store S, bool EXACT>
__global__ void init_f_kernel(Layout L, typename StoreT<S>::T* b0, typename StoreT<S>::T* b1, const double* u,
                              const double* v, const double* w, const double* p, double p_shift, Encoding enc) {
  using R = typename StoreT<S>::R;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  const int k = blockIdx.z;
  if (i >= L.ex) return;
  const int64_t c = i + static_cast<int64_t>(L.ex) * (j + static_cast<int64_t>(L.ey) * k);
  const R uu = R(u[c]), vv = R(v[c]), ww = R(w[c]);
  const R pp = p_shift == 0.0 ? R(p[c]) : R(p[c] - p_shift);
  R tp3[4], udu15;
  feq_prep<R, EXACT>(uu, vv, ww, pp, tp3, udu15);
  const int64_t b = L.idx(0, i, j, k);
  static_for<0, Q>([&](auto qc) {
    constexpr int q = decltype(qc)::value;
    const auto val = encode<S>(feq_of<q, R, EXACT>(uu, vv, ww, tp3, udu15), q, enc);
    b0[b + q * L.sq] = val;
    if (b1) b1[b + q * L.sq] = val;
  });
}

// ------------------------------------------------------------ step
// The step is split into a load phase (pull the 27 populations of a cell,
// applying the boundary rule of each link) and a compute phase (moments,
// case rules, collision, stores).  A thread handles CPT cells stacked along
// y and issues the loads of all of them before any arithmetic, so enough
// bytes are in flight per thread for the narrow storage formats.  Every
// boundary rule is expressed as a per-link choice of source address, never
// as divergent control flow: a warp always issues its loads back to back.

// Cell flags for the standard boundaries: which walls the cell touches
// (bit 0..5: x-, x+, y-, y+, z-, z+) -- the lid is z+.
__device__ __forceinline__ unsigned wall_flags(const StepArgs& a, int i, int j, int k) {
  return (i == 0 ? 1u : 0u) | (i == a.nx - 1 ? 2u : 0u) | (j == 0 ? 4u : 0u) | (j == a.ny - 1 ? 8u : 0u) |
         (k == 0 ? 16u : 0u) | (k == a.nz - 1 ? 32u : 0u);
}
// the link of population q leaves the box through a wall the cell touches
template <int q>
__device__ __forceinline__ bool leaves(unsigned w) {
  constexpr int ex = D3Q27::ex[q], ey = D3Q27::ey[q], ez = D3Q27::ez[q];
  constexpr unsigned m = (ex > 0 ? 1u : 0u) | (ex < 0 ? 2u : 0u) | (ey > 0 ? 4u : 0u) | (ey < 0 ? 8u : 0u) |
                         (ez > 0 ? 16u : 0u) | (ez < 0 ? 32u : 0u);
  return (w & m) != 0u;
}

template <Store S, Bc B, CaseRule RULE, bool EXACT, bool DRAG>
__device__ __forceinline__ void load_cell(const StepArgs& a, const int i, const int j, const int k,
                                          typename StoreT<S>::R (&f)[Q], double (&drag)[3]) {
  using R = typename StoreT<S>::R;
  using T = typename StoreT<S>::T;
  const T* __restrict__ src = static_cast<const T*>(a.src);
  const int64_t b = a.base + k * a.sz + j * a.pitch + i;
  if constexpr (B == Bc::Ghost) {
    // reference boundaries: the ghost slots the pull reaches were filled by
    // the ghost-slot gather after the previous step
    static_for<0, Q>([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      f[q] = decode<S>(ldg_stream(src + b + a.off[q]), q, a.enc);
    });
  } else if constexpr (B == Bc::Periodic) {
    const int im = i == 0 ? a.nx - 1 : i - 1, ip = i == a.nx - 1 ? 0 : i + 1;
    const int jm = j == 0 ? a.ny - 1 : j - 1, jp = j == a.ny - 1 ? 0 : j + 1;
    const int km = k == 0 ? a.nz - 1 : k - 1, kp = k == a.nz - 1 ? 0 : k + 1;
    const int64_t rz[3] = {km * a.sz, k * a.sz, kp * a.sz};
    const int64_t ry[3] = {jm * a.pitch, j * a.pitch, jp * a.pitch};
    const int64_t cx[3] = {im, i, ip};
    static_for<0, Q>([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      const int64_t s = a.base + q * a.sq + rz[1 - D3Q27::ez[q]] + ry[1 - D3Q27::ey[q]] + cx[1 - D3Q27::ex[q]];
      f[q] = decode<S>(ldg_stream(src + s), q, a.enc);
    });
  } else if constexpr (RULE == CaseRule::CavityStd) {
    // halfway bounce-back on the six walls: a link leaving the box returns
    // the cell's own opposite population; through the lid (z+) it gains
    // -2 w rho_w (c_bb . u_w)/cs^2 = 6 w rho_w e_q.u_w
    const unsigned wf = wall_flags(a, i, j, k);
    const bool lid = (wf & 32u) != 0u;
    static_for<0, Q>([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      constexpr int qb = D3Q27::bb[q];
      constexpr int exq = D3Q27::ex[q];
      constexpr int cls = D3Q27::wclass[q];
      const bool out = leaves<q>(wf);
      const int64_t o = out ? static_cast<int64_t>(qb) * a.sq : a.off[q];
      R val = decode<S>(ldg_stream(src + b + o), out ? qb : q, a.enc);
      if constexpr (exq != 0 && D3Q27::ez[q] < 0) {
        // ((6 rho_w u_w) w_q) e_q rounded on its own, then added (EXACT keeps
        // the multiply and the add apart, as the specification does)
        using A = Ar<R, EXACT>;
        if (lid) val = A::add(val, A::mul(A::mul(R(6.0 * a.rho_w * a.lid_u), wgt<R>(cls)), R(exq)));
      }
      f[q] = val;
    });
  } else {
    static_assert(RULE == CaseRule::SphereStd, "standard rule");
    // channel periodic in y and z; x-: equilibrium inlet; x+: zero-gradient
    // outlet (the link re-enters from the cell's own column); solid links
    // (bit q of the cell's link mask) bounce back
    const int jm = j == 0 ? a.ny - 1 : j - 1, jp = j == a.ny - 1 ? 0 : j + 1;
    const int km = k == 0 ? a.nz - 1 : k - 1, kp = k == a.nz - 1 ? 0 : k + 1;
    const int64_t rz[3] = {km * a.sz, k * a.sz, kp * a.sz};
    const int64_t ry[3] = {jm * a.pitch, j * a.pitch, jp * a.pitch};
    const bool inlet = i == 0, outlet = i == a.nx - 1;
    const int64_t cx[3] = {i - 1, i, outlet ? i : i + 1};
    const int64_t cell = i + static_cast<int64_t>(a.nx) * (j + static_cast<int64_t>(a.ny) * k);
    const bool near = k >= a.near_lo[2] && k <= a.near_hi[2] && j >= a.near_lo[1] && j <= a.near_hi[1] &&
                      i >= a.near_lo[0] && i <= a.near_hi[0];
    const uint32_t links = near ? a.links[cell] : 0u;
    static_for<0, Q>([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      constexpr int qb = D3Q27::bb[q];
      constexpr int ex = D3Q27::ex[q], ey = D3Q27::ey[q], ez = D3Q27::ez[q];
      [[maybe_unused]] constexpr int cls = D3Q27::wclass[q];
      const bool solid = (links >> q) & 1u;
      const int64_t s_pull = a.base + q * a.sq + rz[1 - ez] + ry[1 - ey] + cx[1 - ex];
      const int64_t s_bb = b + static_cast<int64_t>(qb) * a.sq;
      R val = decode<S>(ldg_stream(src + (solid ? s_bb : s_pull)), solid ? qb : q, a.enc);
      if constexpr (ex > 0) {
        if (inlet) val = R(a.feq_in[q]);
      }
      if constexpr (DRAG) {
        if (solid) {
          const double fd = static_cast<double>(val) + (S == Store::F64 ? 0.0 : 3.0 * wgt<double>(cls) * a.p_shift);
          if constexpr (ex != 0) drag[0] -= 2.0 * fd * ex;
          if constexpr (ey != 0) drag[1] -= 2.0 * fd * ey;
          if constexpr (ez != 0) drag[2] -= 2.0 * fd * ez;
        }
      }
      f[q] = val;
    });
  }
}

template <Store S, CaseRule RULE, bool EXACT>
__device__ __forceinline__ void compute_cell(const StepArgs& a, const int i, const int j, const int k,
                                             typename StoreT<S>::R (&f)[Q]) {
  using T = typename StoreT<S>::T;
  using R = typename StoreT<S>::R;
  T* __restrict__ dst = static_cast<T*>(a.dst);
  const int64_t b = a.base + k * a.sz + j * a.pitch + i;
  const int64_t cell = i + static_cast<int64_t>(a.nx) * (j + static_cast<int64_t>(a.ny) * k);

  R u, v, w, p;
  moments<R, EXACT>(f, u, v, w, p);

  if constexpr (RULE == CaseRule::CavityRef) {
    // lid_driven_cavity/src/lbm.cpp:343-344: ua forced on the top plane
    if (k == a.nz - 1) u = R(a.lid_u);
  } else if constexpr (RULE == CaseRule::SphereRef) {
    // sphere/src/lbm.cpp:399-412: moments times the mask, then the inlet
    // velocity on the first plane and zero pressure on the last
    if (!a.usr[cell]) {
      u = R(0);
      v = R(0);
      w = R(0);
      p = R(-a.p_shift);
    }
    if (i == 0) {
      u = R(a.inlet[k]);
      v = R(0);
      w = R(0);
    }
    if (i == a.nx - 1) p = R(-a.p_shift);
  }

  if (a.store) {
    a.mu[cell] = u;
    a.mv[cell] = v;
    a.mw[cell] = w;
    a.mp[cell] = static_cast<double>(p) + a.p_shift;
  }

  R tp3[4], udu15;
  feq_prep<R, EXACT>(u, v, w, p, tp3, udu15);
  using A = Ar<R, EXACT>;
  static_for<0, Q>([&](auto qc) {
    constexpr int q = decltype(qc)::value;
    const R feq = feq_of<q, R, EXACT>(u, v, w, tp3, udu15);
    R fs;
    if constexpr (EXACT) {
      fs = A::sub(f[q], __ddiv_rn(A::sub(f[q], feq), a.tau_half));
    } else {
      fs = f[q] - R(a.omega) * (f[q] - feq);
    }
    dst[b + q * a.sq] = encode<S>(fs, q, a.enc);
  });
}

template <Store S> struct CellsPerThread { static constexpr int value = 1; };
template <> struct CellsPerThread<Store::F32> { static constexpr int value = 2; };
template <> struct CellsPerThread<Store::F16> { static constexpr int value = 2; };
template <> struct CellsPerThread<Store::BF16> { static constexpr int value = 2; };

template <Store S, Bc B, CaseRule RULE, bool EXACT, bool DRAG>
__global__ void __launch_bounds__(256, 2) step_kernel(const StepArgs a) {
  using R = typename StoreT<S>::R;
  constexpr int CPT = CellsPerThread<S>::value;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j0 = (blockIdx.y * blockDim.y + threadIdx.y) * CPT;
  const int k = blockIdx.z;
  double drag[3] = {0.0, 0.0, 0.0};
  R f[CPT][Q];
  bool act[CPT];
#pragma unroll
  for (int c = 0; c < CPT; ++c) {
    const int j = j0 + c;
    act[c] = i < a.nx && j < a.ny;
    if constexpr (RULE == CaseRule::SphereStd) {
      // solid cells are not updated; they report zero moments
      if (act[c]) {
        const int64_t cell = i + static_cast<int64_t>(a.nx) * (j + static_cast<int64_t>(a.ny) * k);
        if (!a.usr[cell]) {
          if (a.store) {
            a.mu[cell] = 0;
            a.mv[cell] = 0;
            a.mw[cell] = 0;
            a.mp[cell] = a.p_shift;
          }
          act[c] = false;
        }
      }
    }
    if (act[c]) load_cell<S, B, RULE, EXACT, DRAG>(a, i, j, k, f[c], drag);
  }
#pragma unroll
  for (int c = 0; c < CPT; ++c)
    if (act[c]) compute_cell<S, RULE, EXACT>(a, i, j0 + c, k, f[c]);

  if constexpr (DRAG) {
    // every thread reaches the block reduction; the per-block partial sums
    // are added in a fixed order afterwards, so the force is deterministic
    __shared__ double sh[3][8];
    const int t = threadIdx.x + blockDim.x * threadIdx.y;
    const int lane = t & 31, warp = t >> 5;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      double x = drag[c];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
      if (lane == 0) sh[c][warp] = x;
    }
    __syncthreads();
    if (t < 3) {
      const int nw = (blockDim.x * blockDim.y + 31) / 32;
      double x = 0.0;
      for (int w = 0; w < nw; ++w) x += sh[t][w];
      const int64_t blk = blockIdx.x + static_cast<int64_t>(gridDim.x) * (blockIdx.y + static_cast<int64_t>(gridDim.y) * blockIdx.z);
      a.drag_part[3 * blk + t] = x;
    }
  }
}

// Sum the per-block drag partials (3 components, fixed order).
__global__ void drag_sum_kernel(const double* part, int64_t nblk, double* out) {
  const int c = blockIdx.x;  // component
  double acc = 0.0;
  for (int64_t b = threadIdx.x; b < nblk; b += blockDim.x) acc += part[3 * b + c];
  __shared__ double sh[RED_THREADS_DRAG / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double x = 0.0;
    for (int w = 0; w < RED_THREADS_DRAG / 32; ++w) x += sh[w];
    out[c] = x;
  }
}

// ------------------------------------------------------------ ghost slots
template <Store S>
__global__ void ghost_gather_kernel(typename StoreT<S>::T* __restrict__ dst, const typename StoreT<S>::T* __restrict__ prev,
                                    const int64_t* __restrict__ tgt, const int64_t* __restrict__ src, int64_t n,
                                    int64_t sq, Encoding enc) {
  using T = typename StoreT<S>::T;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < n;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t s = src[e];
    const int64_t t = tgt[e];
    T val;
    if (s >= 0) {
      val = dst[s];
    } else if (s <= -2) {
      val = prev[-s - 2];
    } else {
      val = encode<S>(typename StoreT<S>::R(0), static_cast<int>(t / sq), enc);
    }
    dst[t] = val;
  }
}

// ------------------------------------------------------------ reductions
constexpr int RED_THREADS = 256;
constexpr int RED_BLOCKS = 592;  // 4 per SM on 148 SMs

__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}
__device__ __forceinline__ double warp_max(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_xor_sync(0xffffffffu, x, o));
  return x;
}

// Pass 1: each block reduces a fixed slice of cells (deterministic order) and
// writes one partial; pass 2: one block reduces the partials.
__global__ void reduce_pass1(RedKind kind, const double* u, const double* v, const double* w, const double* p,
                             const double* u2, const double* v2, const double* w2, int64_t n, double* part) {
  double acc = 0.0;
  for (int64_t c = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; c < n;
       c += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double x;
    switch (kind) {
      case RedKind::Mass: x = 3.0 * p[c]; break;
      case RedKind::Kinetic: x = 0.5 * (u[c] * u[c] + v[c] * v[c] + w[c] * w[c]); break;
      case RedKind::DiffSq: {
        const double du = u[c] - u2[c], dv = v[c] - v2[c], dw = w[c] - w2[c];
        x = du * du + dv * dv + dw * dw;
        break;
      }
      case RedKind::NormSq: x = u[c] * u[c] + v[c] * v[c] + w[c] * w[c]; break;
      default: x = sqrt(u[c] * u[c] + v[c] * v[c] + w[c] * w[c]); break;
    }
    acc = kind == RedKind::UMax ? fmax(acc, x) : acc + x;
  }
  __shared__ double sh[RED_THREADS / 32];
  acc = kind == RedKind::UMax ? warp_max(acc) : warp_sum(acc);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    double x = threadIdx.x < RED_THREADS / 32 ? sh[threadIdx.x] : 0.0;
    x = kind == RedKind::UMax ? warp_max(x) : warp_sum(x);
    if (threadIdx.x == 0) part[blockIdx.x] = x;
  }
}

__global__ void reduce_pass2(RedKind kind, const double* part, int nparts, double* out) {
  double acc = 0.0;
  for (int c = threadIdx.x; c < nparts; c += blockDim.x) acc = kind == RedKind::UMax ? fmax(acc, part[c]) : acc + part[c];
  __shared__ double sh[RED_THREADS / 32];
  acc = kind == RedKind::UMax ? warp_max(acc) : warp_sum(acc);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    double x = threadIdx.x < RED_THREADS / 32 ? sh[threadIdx.x] : 0.0;
    x = kind == RedKind::UMax ? warp_max(x) : warp_sum(x);
    if (threadIdx.x == 0) *out = x;
  }
}

}  // namespace

dim3 step_block(int nx) {
  if (nx >= 128) return dim3(128, 2, 1);
  if (nx >= 64) return dim3(64, 4, 1);
  return dim3(32, 8, 1);
}

// ------------------------------------------------------------ launchers
int reduce_blocks() { return RED_BLOCKS; }

int64_t step_grid_blocks(int nx, int ny, int nz, int storage) {
  const dim3 b = step_block(nx);
  const int cpt = storage == static_cast<int>(Store::F64) ? 1 : CellsPerThread<Store::F16>::value;
  const int rows = b.y * cpt;
  return static_cast<int64_t>((nx + b.x - 1) / b.x) * ((ny + rows - 1) / rows) * nz;
}

cudaError_t launch_drag_sum(const double* part, int64_t nblk, double* out, cudaStream_t s) {
  drag_sum_kernel<<<3, RED_THREADS_DRAG, 0, s>>>(part, nblk, out);
  return cudaGetLastError();
}

cudaError_t launch_reduce(RedKind k, const double* u, const double* v, const double* w, const double* p,
                          const double* u2, const double* v2, const double* w2, int64_t n, double* scratch,
                          double* out, cudaStream_t s) {
  reduce_pass1<<<RED_BLOCKS, RED_THREADS, 0, s>>>(k, u, v, w, p, u2, v2, w2, n, scratch);
  reduce_pass2<<<1, RED_THREADS, 0, s>>>(k, scratch, RED_BLOCKS, out);
  return cudaGetLastError();
}

template <Store S, bool EXACT>
static cudaError_t init_f_impl(const Layout& L, void* b0, void* b1, const double* u, const double* v,
                               const double* w, const double* p, double p_shift, const Encoding& enc,
                               cudaStream_t s) {
  using T = typename StoreT<S>::T;
  dim3 block(128, 1, 1);
  dim3 grid((L.ex + 127) / 128, L.ey, L.ez);
  init_f_kernel<S, EXACT><<<grid, block, 0, s>>>(L, static_cast<T*>(b0), static_cast<T*>(b1), u, v, w, p, p_shift,
                                                 enc);
  return cudaGetLastError();
}

cudaError_t launch_init_f(const LaunchCfg& c, const Layout& L, void* buf0, void* buf1, const double* u,
                          const double* v, const double* w, const double* p, double p_shift, const Encoding& enc,
                          cudaStream_t s) {
  switch (c.store) {
    case Store::F64:
      return c.exact ? init_f_impl<Store::F64, true>(L, buf0, buf1, u, v, w, p, 0.0, enc, s)
                     : init_f_impl<Store::F64, false>(L, buf0, buf1, u, v, w, p, 0.0, enc, s);
    case Store::F32: return init_f_impl<Store::F32, false>(L, buf0, buf1, u, v, w, p, p_shift, enc, s);
    case Store::F16: return init_f_impl<Store::F16, false>(L, buf0, buf1, u, v, w, p, p_shift, enc, s);
    case Store::BF16: return init_f_impl<Store::BF16, false>(L, buf0, buf1, u, v, w, p, p_shift, enc, s);
  }
  return cudaErrorInvalidValue;
}

template <Store S, Bc B, CaseRule R, bool EXACT>
static cudaError_t step_impl(const StepArgs& a, cudaStream_t s) {
  const dim3 block = step_block(a.nx);
  const int rows = block.y * CellsPerThread<S>::value;
  const dim3 grid((a.nx + block.x - 1) / block.x, (a.ny + rows - 1) / rows, a.nz);
  if constexpr (R == CaseRule::SphereStd) {
    if (a.drag_part) {
      step_kernel<S, B, R, EXACT, true><<<grid, block, 0, s>>>(a);
      return cudaGetLastError();
    }
  }
  step_kernel<S, B, R, EXACT, false><<<grid, block, 0, s>>>(a);
  return cudaGetLastError();
}

template <Store S, bool EXACT>
static cudaError_t step_rule(const LaunchCfg& c, const StepArgs& a, cudaStream_t s) {
  switch (c.rule) {
    case CaseRule::None: return step_impl<S, Bc::Periodic, CaseRule::None, EXACT>(a, s);
    case CaseRule::CavityRef: return step_impl<S, Bc::Ghost, CaseRule::CavityRef, EXACT>(a, s);
    case CaseRule::SphereRef: return step_impl<S, Bc::Ghost, CaseRule::SphereRef, EXACT>(a, s);
    case CaseRule::CavityStd: return step_impl<S, Bc::Standard, CaseRule::CavityStd, EXACT>(a, s);
    case CaseRule::SphereStd: return step_impl<S, Bc::Standard, CaseRule::SphereStd, EXACT>(a, s);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_step(const LaunchCfg& c, const StepArgs& a, cudaStream_t s) {
  switch (c.store) {
    case Store::F64: return c.exact ? step_rule<Store::F64, true>(c, a, s) : step_rule<Store::F64, false>(c, a, s);
    case Store::F32: return step_rule<Store::F32, false>(c, a, s);
    case Store::F16: return step_rule<Store::F16, false>(c, a, s);
    case Store::BF16: return step_rule<Store::BF16, false>(c, a, s);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_ghost_gather(Store st, void* dst, const void* prev, const int64_t* tgt, const int64_t* src,
                                int64_t n, int64_t sq, const Encoding& enc, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const int threads = 256;
  const int64_t want = (n + threads - 1) / threads;
  const int blocks = static_cast<int>(want < 148 * 16 ? want : 148 * 16);
  switch (st) {
#define IMX_GG(S)                                                                                            \
  case S:                                                                                                    \
    ghost_gather_kernel<S><<<blocks, threads, 0, s>>>(static_cast<typename StoreT<S>::T*>(dst),            \
                                                     static_cast<const typename StoreT<S>::T*>(prev), tgt, \
                                                     src, n, sq, enc);                                     \
    break;
    IMX_GG(Store::F64)
    IMX_GG(Store::F32)
    IMX_GG(Store::F16)
    IMX_GG(Store::BF16)
#undef IMX_GG
  }
  return cudaGetLastError();
}

}  // namespace imx
