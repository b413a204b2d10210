// Per-cell device machinery of the fused D3Q27 step, shared by the
// single-lattice kernels (kernels.cu) and the batched engine (engine.cu):
// arithmetic modes, equilibrium, moments, storage encodings, and the load and
// compute phases of one cell.  See kernels.cu for the step's structure.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <type_traits>
#include <utility>

#include "lattice.h"

namespace imx {
namespace core {

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

// RN(x / d) for d > 0, given z = RN(1/d), proven on the fast path and
// deferred to IEEE division otherwise (div_rn_fast, then div_rn_slow):
//   q0 = RN(x z), r0 = x - q0 d (fma), q1 = RN(q0 + r0 z)   (Markstein 1990)
//   r1 = x - q1 d by fma is exact whenever q1 is within one ulp of x/d (the
//   remainder is then an integer multiple of ulp(q1) ulp(d) below 2^53 of them);
//   q1 is the correctly rounded quotient if x/d lies strictly within half the
//   smaller neighbouring gap of q1, i.e. |r1| < d * gap_below(q1) / 2.  If q1 is
//   further than one ulp away, |r1| exceeds that bound, so a wrong q1 is never
//   accepted; rejected cases (ties, near-ties, tiny quotients) take
//   __ddiv_rn.  The bound is a power of two times d, so it is exact.  The test
//   reads only the high word of q1: when its 20 high significand bits are not
//   all zero q1 is no power of two, gap_below(q1) = ulp(q1) and the bound is
//   d * 2^(E - 53), E the exponent of q1; the other quotients (a 2^-20
//   fraction, powers of two among them) take __ddiv_rn.
//   A zero numerator is returned as it is (IEEE: +-0 / d = +-0 for d > 0); it
//   is common (a cell at rest has f = feq).  div_rn_fast is this fast path:
//   *q is RN(x / d) when it returns true; otherwise the caller finishes with
//   div_rn_slow, which also returns an infinite numerator (+-inf / d = +-inf)
//   and a NaN (the quotient is NaN) of a lattice that overflowed as they are.
//   Branch-free, so that the collision's 27 divisions form one straight run
//   of code.
__device__ __forceinline__ bool div_rn_fast(double x, double d, double z, double* q) {
  const double q0 = __dmul_rn(x, z);
  const double r0 = __fma_rn(-q0, d, x);
  const double q1 = __fma_rn(r0, z, q0);
  const double r1 = __fma_rn(-q1, d, x);
  const int hi = __double2hiint(q1);
  const int he = (hi & 0x7ff00000) - (53 << 20);
  const bool ok = he > 0 && (hi & 0x000fffff) != 0 && fabs(r1) < __dmul_rn(d, __hiloint2double(he, 0));
  const bool zero = x == 0.0;
  *q = zero ? x : q1;
  return ok || zero;
}

// The cases div_rn_fast leaves: non-finite numerators (returned as they
// are) and the rest through IEEE division.
__device__ __forceinline__ double div_rn_slow(double x, double d) { return isfinite(x) ? __ddiv_rn(x, d) : x; }

// Populations per redo group of the EXACT collision (a divisor of 27): the
// fast quotients of a group form one straight run of code, and the group's
// f values stay live until its redo check.
constexpr int EXACT_GROUP = 3;

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

// ------------------------------------------------------------ stochastic rounding
// With stochastic rounding (Encoding::sr; the cavity's and the sphere's
// 2-byte formats) the stores convert with sm_100a's `cvt.rs` (PTX ISA 8.7:
// FP32 to f16x2 / bf16x2 rounded stochastically with caller-given random
// bits), so a value rounds up with probability equal to its distance from
// the one below and the rounding error is zero on average (stochastic
// rounding: Forsythe 1959; Connolly, Higham and Mary, SIAM J. Sci. Comput.
// 43, 2021).  In a steady flow round-to-nearest makes the same error at the
// same cell every step, a constant forcing whose effect on the velocity
// grows with the step count; zero-mean errors do not accumulate that way.
// The random bits are a function of (cell, population, step) only, so a
// lattice gives the same bits alone, in the engine and resumed from a
// checkpoint: per cell (or x-pair) x = sr_hash(cell index ^ seed), with
// StepArgs::seed the hash of the lattice's step count (sr_hash: lattice.h),
// and population q takes the 32 bits of x * sr_mul(q).
constexpr uint32_t sr_mul(int q) { return 0x9e3779b9u * (2u * static_cast<uint32_t>(q) + 1u) | 1u; }
// An x-pair of FP32 values (lo = cell x0) to the 2-byte format's packed
// pair, rounded stochastically with the 32 random bits `rbits`.
template <Store S>
__device__ __forceinline__ uint32_t sr_pair(float2 g, uint32_t rbits) {
  uint32_t word;
  if constexpr (S == Store::F16)
    asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(word) : "f"(g.y), "f"(g.x), "r"(rbits));
  else
    asm("cvt.rs.bf16x2.f32 %0, %1, %2, %3;" : "=r"(word) : "f"(g.y), "f"(g.x), "r"(rbits));
  return word;
}
// One FP32 value, the same way (the low half of a pair whose high half is 0).
template <Store S>
__device__ __forceinline__ typename StoreT<S>::T sr_one(float x, uint32_t rbits) {
  const unsigned short h = static_cast<unsigned short>(sr_pair<S>(make_float2(x, 0.f), rbits) & 0xffffu);
  if constexpr (S == Store::F16)
    return __ushort_as_half(h);
  else
    return __ushort_as_bfloat16(h);
}

template <class T>
__device__ __forceinline__ T ldg_stream(const T* p) {
  return __ldg(p);
}

// ------------------------------------------------------------ step
// The step is split into a load phase (pull the 27 populations of a cell,
// applying the boundary rule of each link) and a compute phase (moments,
// case rules, collision, stores).  A thread handles CPT cells stacked along
// y and issues the loads of all of them before any arithmetic, so enough
// bytes are in flight per thread for the narrow storage formats.  Every
// boundary rule is expressed as a per-link choice of source address, never
// as divergent control flow: a warp always issues its loads back to back.
//
// Addressing: each population q lives in its own plane; a cell's value is
// plane_q[idx] with idx = base + k*sz + j*pitch + i (32-bit, in elements),
// and the pull adds the plane-independent offset rel[q] = -(ez sz + ey pitch
// + ex).  The single-lattice kernels take the 27 plane pointers as launch
// parameters; the engine derives them from one buffer and the plane stride.

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

// Population planes of the source and destination buffers.
template <class T>
struct Planes {
  const T* const* srcq;  // 27 source plane pointers
  T* const* dstq;        // 27 destination plane pointers
  __device__ __forceinline__ T load(int q, int32_t idx) const { return ldg_stream(srcq[q] + idx); }
  __device__ __forceinline__ void store(int q, int32_t idx, T v) const { dstq[q][idx] = v; }
  // x-pair formats: an aligned pair (idx even) or one value, as raw bits
  // (32-bit pairs of 16-bit values; FP32: 64-bit pairs of 32-bit values)
  using W = std::conditional_t<sizeof(T) == 4, uint2, uint32_t>;
  using H = std::conditional_t<sizeof(T) == 4, uint32_t, uint16_t>;
  __device__ __forceinline__ W load_pair(int q, int32_t idx) const {
    return __ldg(reinterpret_cast<const W*>(srcq[q] + idx));
  }
  __device__ __forceinline__ uint32_t load_half(int q, int32_t idx) const {
    return __ldg(reinterpret_cast<const unsigned short*>(srcq[q] + idx));
  }
  __device__ __forceinline__ void store_pair(int q, int32_t idx, W v) const {
    *reinterpret_cast<W*>(dstq[q] + idx) = v;
  }
  __device__ __forceinline__ void store_half(int q, int32_t idx, H v) const { *reinterpret_cast<H*>(dstq[q] + idx) = v; }
};

// Population planes at one stride: plane q starts q * sq elements into the
// buffer.  A thread's per-cell index is one 64-bit address; each
// population's offset q * sq is the same for every thread of the block (the
// shared-memory staged kernels, whose reads come from the stage and whose
// stores go here).
template <class T>
struct StridedPlanes {
  const T* src;
  T* dst;
  int64_t sq;
  using W = std::conditional_t<sizeof(T) == 4, uint2, uint32_t>;
  using H = std::conditional_t<sizeof(T) == 4, uint32_t, uint16_t>;
  __device__ __forceinline__ T load(int q, int32_t idx) const { return ldg_stream(src + idx + q * sq); }
  __device__ __forceinline__ void store(int q, int32_t idx, T v) const { dst[idx + q * sq] = v; }
  __device__ __forceinline__ W load_pair(int q, int32_t idx) const {
    return __ldg(reinterpret_cast<const W*>(src + idx + q * sq));
  }
  __device__ __forceinline__ uint32_t load_half(int q, int32_t idx) const {
    return __ldg(reinterpret_cast<const unsigned short*>(src + idx + q * sq));
  }
  __device__ __forceinline__ void store_pair(int q, int32_t idx, W v) const {
    *reinterpret_cast<W*>(dst + idx + q * sq) = v;
  }
  __device__ __forceinline__ void store_half(int q, int32_t idx, H v) const {
    *reinterpret_cast<H*>(dst + idx + q * sq) = v;
  }
};

template <Store S, Bc B, CaseRule RULE, bool EXACT, bool DRAG, class P>
__device__ __forceinline__ void load_cell(const StepArgs& a, const P& pl, const int i, const int j, const int k,
                                          typename StoreT<S>::R (&f)[Q], double (&drag)[3]) {
  using R = typename StoreT<S>::R;
  const int32_t b = a.base32 + k * a.sz32 + j * a.pitch32 + i;
  if constexpr (B == Bc::Ghost) {
    if constexpr (RULE == CaseRule::CavityRef) {
      const unsigned wf = a.face_codes ? wall_flags(a, i, j, k) : 0u;
      if (wf != 0u) {
        // a face cell of the reference cavity, with the boundary passes
        // resolved per link (the face-code table, lattice.h): its 28 code
        // words in seven 16-byte loads, the pull address of every link that
        // leaves the box replaced, then all 27 value loads at once.  Only
        // the face blocks of the step grid reach here (step_kernel), so no
        // warp mixes this path with the inside cells' one.
        using T = typename StoreT<S>::T;
        const int face = __ffs(static_cast<int>(wf)) - 1;
        const int fa = face < 2 ? j : i, fb = face < 4 ? k : j;
        const int4* cw = reinterpret_cast<const int4*>(
            a.face_codes + a.face_base[face] + (static_cast<int64_t>(fb) * a.face_dim[face] + fa) * FACE_CODE_WORDS);
        int32_t code[FACE_CODE_WORDS];
#pragma unroll
        for (int v = 0; v < FACE_CODE_WORDS / 4; ++v) {
          const int4 c4 = __ldg(cw + v);
          code[4 * v] = c4.x;
          code[4 * v + 1] = c4.y;
          code[4 * v + 2] = c4.z;
          code[4 * v + 3] = c4.w;
        }
        const T* in = static_cast<const T*>(a.src);
        const T* out = static_cast<const T*>(a.dst);  // ghost slots only: this step writes the interior
        T raw[Q];
        static_for<0, Q>([&](auto qc) {
          constexpr int q = decltype(qc)::value;
          const T* ptr = pl.srcq[q] + (b + a.rel[q]);
          if (leaves<q>(wf)) {
            const int32_t c = code[q];
            ptr = c >= 0 ? in + c : (c == -1 ? ptr : out + (-static_cast<int64_t>(c) - 2));
          }
          raw[q] = __ldg(ptr);
        });
        const uint32_t keep = static_cast<uint32_t>(code[Q]);
        static_for<0, Q>([&](auto qc) {
          constexpr int q = decltype(qc)::value;
          if (leaves<q>(wf)) {
            if (code[q] == -1) raw[q] = T(0);
            // the value a later step reads as this slot's previous one
            if ((keep >> q) & 1u) const_cast<T*>(in)[q * a.sq + b + a.rel[q]] = raw[q];
          }
          f[q] = decode<S>(raw[q], q, a.enc);
        });
        return;
      }
    }
    // reference boundaries: the ghost slots the pull reaches were filled by
    // the ghost-slot gather after the previous step (or the cell is inside)
    static_for<0, Q>([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      f[q] = decode<S>(pl.load(q, b + a.rel[q]), q, a.enc);
    });
  } else if constexpr (B == Bc::Periodic) {
    const int im = i == 0 ? a.nx - 1 : i - 1, ip = i == a.nx - 1 ? 0 : i + 1;
    const int jm = j == 0 ? a.ny - 1 : j - 1, jp = j == a.ny - 1 ? 0 : j + 1;
    const int km = k == 0 ? a.nz - 1 : k - 1, kp = k == a.nz - 1 ? 0 : k + 1;
    const int32_t rz[3] = {a.base32 + km * a.sz32, a.base32 + k * a.sz32, a.base32 + kp * a.sz32};
    const int32_t ry[3] = {jm * a.pitch32, j * a.pitch32, jp * a.pitch32};
    const int32_t cx[3] = {im, i, ip};
    static_for<0, Q>([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      const int32_t s = rz[1 - D3Q27::ez[q]] + ry[1 - D3Q27::ey[q]] + cx[1 - D3Q27::ex[q]];
      f[q] = decode<S>(pl.load(q, s), q, a.enc);
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
      // q and bb(q) share the weight class, hence the storage scale
      R val = decode<S>(out ? pl.load(qb, b) : pl.load(q, b + a.rel[q]), q, a.enc);
      if constexpr (exq != 0 && D3Q27::ez[q] < 0) {
        // ((6 rho_w u_w) w_q) e_q rounded on its own, then added (EXACT keeps
        // the multiply and the add apart, as the specification does)
        using A = Ar<R, EXACT>;
        if (lid) val = A::add(val, A::mul(A::mul(R(6.0 * a.rho_w * a.lid_u), wgt<R>(cls)), R(exq)));
      }
      f[q] = val;
    });
  } else if constexpr (RULE == CaseRule::SlabStd) {
    // x and y periodic; halfway bounce-back through the bottom (z-, at rest)
    // and the lid (z+, moving: the same term as the cavity's lid)
    const int im = i == 0 ? a.nx - 1 : i - 1, ip = i == a.nx - 1 ? 0 : i + 1;
    const int jm = j == 0 ? a.ny - 1 : j - 1, jp = j == a.ny - 1 ? 0 : j + 1;
    const int32_t ry[3] = {jm * a.pitch32, j * a.pitch32, jp * a.pitch32};
    const int32_t cx[3] = {im, i, ip};
    const int32_t rz = a.base32 + k * a.sz32;
    const bool bottom = k == 0, lid = k == a.nz - 1;
    static_for<0, Q>([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      constexpr int qb = D3Q27::bb[q];
      constexpr int exq = D3Q27::ex[q], eyq = D3Q27::ey[q], ezq = D3Q27::ez[q];
      constexpr int cls = D3Q27::wclass[q];
      const bool out = (ezq > 0 && bottom) || (ezq < 0 && lid);
      // the pulled address only where the link stays inside (k - e_z is a plane)
      const int32_t s_pull = out ? b : rz - ezq * a.sz32 + ry[1 - eyq] + cx[1 - exq];
      R val = decode<S>(out ? pl.load(qb, b) : pl.load(q, s_pull), q, a.enc);
      if constexpr (exq != 0 && ezq < 0) {
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
    const int32_t rz[3] = {a.base32 + km * a.sz32, a.base32 + k * a.sz32, a.base32 + kp * a.sz32};
    const int32_t ry[3] = {jm * a.pitch32, j * a.pitch32, jp * a.pitch32};
    const bool inlet = i == 0, outlet = i == a.nx - 1;
    const int32_t cx[3] = {i - 1, i, outlet ? i : i + 1};
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
      const int32_t s_pull = rz[1 - ez] + ry[1 - ey] + cx[1 - ex];
      R val = decode<S>(solid ? pl.load(qb, b) : pl.load(q, s_pull), q, a.enc);
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

// Moment rules of the reference cases, applied to one cell's moments.
template <CaseRule RULE, class R>
__device__ __forceinline__ void case_rules(const StepArgs& a, const int i, const int k, const int64_t cell, R& u,
                                           R& v, R& w, R& p) {
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
}

template <Store S, CaseRule RULE, bool EXACT, class P>
__device__ __forceinline__ void compute_cell(const StepArgs& a, const P& pl, const int i, const int j, const int k,
                                             typename StoreT<S>::R (&f)[Q]) {
  using R = typename StoreT<S>::R;
  const int32_t b = a.base32 + k * a.sz32 + j * a.pitch32 + i;
  const int64_t cell = i + static_cast<int64_t>(a.nx) * (j + static_cast<int64_t>(a.ny) * k);

  R u, v, w, p;
  moments<R, EXACT>(f, u, v, w, p);
  case_rules<RULE>(a, i, k, cell, u, v, w, p);

  if (a.store) {
    a.mu[cell] = u;
    a.mv[cell] = v;
    a.mw[cell] = w;
    a.mp[cell] = static_cast<double>(p) + a.p_shift;
  }

  R tp3[4], udu15;
  feq_prep<R, EXACT>(u, v, w, p, tp3, udu15);
  using A = Ar<R, EXACT>;
  if constexpr (EXACT) {
    // f - (f - feq) / (tau0 + 1/2) with a correctly rounded division, in
    // groups of EXACT_GROUP populations: each population of a group through
    // the branch-free fast path and stored; the few the fast path cannot
    // accept (near-ties, tiny or non-finite numerators) are computed again
    // through IEEE division and stored over the first value before the next
    // group starts, so that only one group's f stays live for that pass
    static_for<0, Q / EXACT_GROUP>([&](auto gc) {
      constexpr int g0 = decltype(gc)::value * EXACT_GROUP;
      uint32_t redo = 0u;
      static_for<g0, g0 + EXACT_GROUP>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        const R feq = feq_of<q, R, EXACT>(u, v, w, tp3, udu15);
        double quot;
        if (!div_rn_fast(A::sub(f[q], feq), a.tau_half, a.omega, &quot)) redo |= 1u << q;
        pl.store(q, b, encode<S>(A::sub(f[q], quot), q, a.enc));
      });
      if (redo) {
        static_for<g0, g0 + EXACT_GROUP>([&](auto qc) {
          constexpr int q = decltype(qc)::value;
          if ((redo >> q) & 1u) {
            const R feq = feq_of<q, R, EXACT>(u, v, w, tp3, udu15);
            pl.store(q, b, encode<S>(A::sub(f[q], div_rn_slow(A::sub(f[q], feq), a.tau_half)), q, a.enc));
          }
        });
      }
    });
  } else {
    [[maybe_unused]] bool sr = false;
    [[maybe_unused]] uint32_t x = 0;
    if constexpr ((S == Store::F16 || S == Store::BF16) && RULE != CaseRule::None) {
      sr = a.enc.sr != 0;
      x = sr_hash(static_cast<uint32_t>(cell) ^ a.seed);
    }
    static_for<0, Q>([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      const R feq = feq_of<q, R, EXACT>(u, v, w, tp3, udu15);
      const R fs = f[q] - R(a.omega) * (f[q] - feq);
      if constexpr ((S == Store::F16 || S == Store::BF16) && RULE != CaseRule::None) {
        if (sr) {
          pl.store(q, b, sr_one<S>(fs * a.enc.scale[q], x * sr_mul(q)));
          return;
        }
      }
      pl.store(q, b, encode<S>(fs, q, a.enc));
    });
  }
}

// Two cells at once in FP32 with Blackwell's paired FP32 instructions: every
// operation of the collision acts on the same quantity of both cells, so the
// pair costs about the instructions of one.  Same arithmetic as
// compute_cell's FP32 path.  The operations are written as PTX
// add/mul/fma.rn.f32x2: an explicit rounding mode forbids the code generator
// to fuse a multiply into a later add, so every kernel that inlines this code
// rounds the same way and their results agree bit for bit (the x-pair
// register kernels, the staged kernels and the engine's).
__device__ __forceinline__ float2 add2rn(float2 a, float2 b) {
  float2 d;
  asm("{\n .reg .b64 ra, rb, rd;\n mov.b64 ra, {%2, %3};\n mov.b64 rb, {%4, %5};\n"
      " add.rn.f32x2 rd, ra, rb;\n mov.b64 {%0, %1}, rd;\n}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return d;
}
__device__ __forceinline__ float2 mul2rn(float2 a, float2 b) {
  float2 d;
  asm("{\n .reg .b64 ra, rb, rd;\n mov.b64 ra, {%2, %3};\n mov.b64 rb, {%4, %5};\n"
      " mul.rn.f32x2 rd, ra, rb;\n mov.b64 {%0, %1}, rd;\n}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return d;
}
__device__ __forceinline__ float2 fma2rn(float2 a, float2 b, float2 c) {
  float2 d;
  asm("{\n .reg .b64 ra, rb, rc, rd;\n mov.b64 ra, {%2, %3};\n mov.b64 rb, {%4, %5};\n"
      " mov.b64 rc, {%6, %7};\n fma.rn.f32x2 rd, ra, rb, rc;\n mov.b64 {%0, %1}, rd;\n}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
  return d;
}
__device__ __forceinline__ float2 sub2rn(float2 a, float2 b) {
  float2 d;
  asm("{\n .reg .b64 ra, rb, rd;\n mov.b64 ra, {%2, %3};\n mov.b64 rb, {%4, %5};\n"
      " sub.rn.f32x2 rd, ra, rb;\n mov.b64 {%0, %1}, rd;\n}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return d;
}
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 f2s(float a) { return make_float2(a, a); }

// e = c_q . u of a pair without negations.  Round-to-nearest is symmetric
// in sign, so (-x) + y rounds to y - x and (-x) + (-y) to -(x + y): the
// value equals the left-to-right sum of the signed components (edu2), or
// its negation when edu_neg<q>() is true; callers fold that sign into the
// constants the value is multiplied by.
template <int q>
constexpr bool edu_neg() {
  constexpr int s[3] = {D3Q27::ex[q], D3Q27::ey[q], D3Q27::ez[q]};
  int sg[3] = {0, 0, 0}, n = 0;
  for (int i = 0; i < 3; ++i)
    if (s[i] != 0) sg[n++] = s[i];
  if (n == 1) return sg[0] < 0;
  if (n == 2) return sg[0] < 0 && sg[1] < 0;
  return n == 3 && sg[0] < 0 && sg[1] < 0 && sg[2] < 0;
}

// s1 x + s2 y for signs s1, s2 = +-1, negated when both are negative
template <int s1, int s2>
__device__ __forceinline__ float2 signed_sum2(float2 x, float2 y) {
  if constexpr (s1 > 0 && s2 > 0) return add2rn(x, y);
  else if constexpr (s1 > 0) return sub2rn(x, y);
  else if constexpr (s2 > 0) return sub2rn(y, x);
  else return add2rn(x, y);
}

template <int q>
__device__ __forceinline__ float2 edu2f(float2 u, float2 v, float2 w) {
  constexpr int a = D3Q27::ex[q], b = D3Q27::ey[q], c = D3Q27::ez[q];
  if constexpr (a != 0 && b != 0 && c != 0) {
    const float2 t = signed_sum2<a, b>(u, v);
    constexpr bool tneg = a < 0 && b < 0;
    if constexpr (!tneg) return c > 0 ? add2rn(t, w) : sub2rn(t, w);
    else return c > 0 ? sub2rn(w, t) : add2rn(t, w);
  } else if constexpr (a != 0 && b != 0) {
    return signed_sum2<a, b>(u, v);
  } else if constexpr (a != 0 && c != 0) {
    return signed_sum2<a, c>(u, w);
  } else if constexpr (b != 0 && c != 0) {
    return signed_sum2<b, c>(v, w);
  } else if constexpr (a != 0) {
    return u;
  } else if constexpr (b != 0) {
    return v;
  } else {
    return w;
  }
}

template <int q>
__device__ __forceinline__ float2 edu2(float2 u, float2 v, float2 w) {
  constexpr int a = D3Q27::ex[q], b = D3Q27::ey[q], c = D3Q27::ez[q];
  float2 t = f2s(0.f);
  bool have = false;
  if constexpr (a != 0) {
    t = a > 0 ? u : f2(-u.x, -u.y);
    have = true;
  }
  if constexpr (b != 0) {
    if (have)
      t = b > 0 ? add2rn(t, v) : add2rn(t, f2(-v.x, -v.y));
    else
      t = b > 0 ? v : f2(-v.x, -v.y);
    have = true;
  }
  if constexpr (c != 0) {
    if (have)
      t = c > 0 ? add2rn(t, w) : add2rn(t, f2(-w.x, -w.y));
    else
      t = c > 0 ? w : f2(-w.x, -w.y);
  }
  return t;
}

template <Store S, CaseRule RULE, class P>
__device__ __forceinline__ void compute_pair(const StepArgs& a, const P& pl, const int i, const int j, const int k,
                                             float (&f0)[Q], float (&f1)[Q]) {
  // cells (i, j, k) and (i, j + 1, k)
  const int32_t b0 = a.base32 + k * a.sz32 + j * a.pitch32 + i;
  const int32_t b1 = b0 + a.pitch32;
  const int64_t c0 = i + static_cast<int64_t>(a.nx) * (j + static_cast<int64_t>(a.ny) * k);
  const int64_t c1 = c0 + a.nx;
  float2 s = f2s(0.f), u = f2s(0.f), v = f2s(0.f), w = f2s(0.f);
  static_for<0, Q>([&](auto qc) {
    constexpr int q = decltype(qc)::value;
    const float2 x = f2(f0[q], f1[q]);
    s = add2rn(s, x);
    if constexpr (D3Q27::ex[q] == 1) u = add2rn(u, x);
    if constexpr (D3Q27::ex[q] == -1) u = sub2rn(u, x);
    if constexpr (D3Q27::ey[q] == 1) v = add2rn(v, x);
    if constexpr (D3Q27::ey[q] == -1) v = sub2rn(v, x);
    if constexpr (D3Q27::ez[q] == 1) w = add2rn(w, x);
    if constexpr (D3Q27::ez[q] == -1) w = sub2rn(w, x);
  });
  float2 p = mul2rn(s, f2s(1.0f / 3.0f));
  case_rules<RULE>(a, i, k, c0, u.x, v.x, w.x, p.x);
  case_rules<RULE>(a, i, k, c1, u.y, v.y, w.y, p.y);
  if (a.store) {
    a.mu[c0] = u.x;
    a.mv[c0] = v.x;
    a.mw[c0] = w.x;
    a.mp[c0] = static_cast<double>(p.x) + a.p_shift;
    a.mu[c1] = u.y;
    a.mv[c1] = v.y;
    a.mw[c1] = w.y;
    a.mp[c1] = static_cast<double>(p.y) + a.p_shift;
  }
  const float2 udu15 = mul2rn(f2s(1.5f), fma2rn(w, w, fma2rn(v, v, mul2rn(u, u))));
  float2 tp3[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) tp3[c] = mul2rn(p, f2s(3.0f * wgt<float>(c)));
  const float2 om = f2s(-static_cast<float>(a.omega));
  static_for<0, Q>([&](auto qc) {
    constexpr int q = decltype(qc)::value;
    constexpr int cls = D3Q27::wclass[q];
    const float2 e = edu2<q>(u, v, w);
    // t (3e + 4.5 e^2 - 1.5 u.u) + 3 t p, with e (3 + 4.5 e) for the bracket
    const float2 br = sub2rn(mul2rn(e, fma2rn(e, f2s(4.5f), f2s(3.0f))), udu15);
    const float2 feq = fma2rn(f2s(wgt<float>(cls)), br, tp3[cls]);
    const float2 x = f2(f0[q], f1[q]);
    const float2 fs = fma2rn(om, sub2rn(x, feq), x);
    pl.store(q, b0, encode<S>(fs.x, q, a.enc));
    pl.store(q, b1, encode<S>(fs.y, q, a.enc));
  });
}

// Rows of x-pairs a thread of the register pair kernels owns: two for the
// 2-byte formats (4-byte pair words), one for FP32 (8-byte pair words), so
// that a thread has 216 bytes of loads in flight either way.
template <Store S> struct PairRows { static constexpr int value = S == Store::F32 ? 1 : 2; };

template <Store S> struct CellsPerThread { static constexpr int value = 1; };
template <> struct CellsPerThread<Store::F32> { static constexpr int value = 2; };
template <> struct CellsPerThread<Store::F16> { static constexpr int value = 2; };
template <> struct CellsPerThread<Store::BF16> { static constexpr int value = 2; };

// The step of the CPT cells (i, j0 .. j0 + CPT - 1, k) a thread owns.
// Returns nothing; writes the next buffer and, with a.store, the moments.
template <Store S, Bc B, CaseRule RULE, bool EXACT, bool DRAG, class P>
__device__ __forceinline__ void step_cells(const StepArgs& a, const P& pl, const int i, const int j0, const int k,
                                           double (&drag)[3]) {
  using R = typename StoreT<S>::R;
  constexpr int CPT = CellsPerThread<S>::value;
  R f[CPT][Q];
  bool act[CPT];
#pragma unroll
  for (int c = 0; c < CPT; ++c) {
    const int j = j0 + c;
    act[c] = i < a.nx && j < a.ny;
    if constexpr (RULE == CaseRule::CavityRef) {
      // with the face blocks (step_kernel), the inside blocks skip face cells
      if (a.face_cells && wall_flags(a, i, j, k) != 0u) act[c] = false;
    }
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
    if (act[c]) load_cell<S, B, RULE, EXACT, DRAG>(a, pl, i, j, k, f[c], drag);
  }
  if constexpr (CPT == 2 && !std::is_same<R, double>::value) {
    if (act[0] && act[1]) {
      compute_pair<S, RULE>(a, pl, i, j0, k, f[0], f[1]);
      return;
    }
  }
#pragma unroll
  for (int c = 0; c < CPT; ++c)
    if (act[c]) compute_cell<S, RULE, EXACT>(a, pl, i, j0 + c, k, f[c]);
}


// ------------------------------------------------------------ 2-byte x-pairs
// For the 2-byte formats a thread owns a 2 x 2 block of cells: the x-pair
// (x0, x0 + 1), x0 even, in rows j0 and j0 + 1.  Every population moves as an
// aligned 4-byte pair, which the paired FP32 instructions then process as one
// float2, so a thread keeps 90 four-byte loads in flight (the 18 populations
// with e_x != 0 take two pairs each, see below).  Needs nx even.

template <Store S> struct Pack2;
template <> struct Pack2<Store::F16> {
  static __device__ __forceinline__ float2 to_f2(uint32_t b) {
    __half2 h = *reinterpret_cast<__half2*>(&b);
    return __half22float2(h);
  }
  static __device__ __forceinline__ uint32_t from_f2(float2 f) {
    __half2 h = __float22half2_rn(f);
    return *reinterpret_cast<uint32_t*>(&h);
  }
  static __device__ __forceinline__ uint16_t from_f(float f) { return __half_as_ushort(__float2half_rn(f)); }
};
template <> struct Pack2<Store::BF16> {
  static __device__ __forceinline__ float2 to_f2(uint32_t b) {
    __nv_bfloat162 h = *reinterpret_cast<__nv_bfloat162*>(&b);
    return __bfloat1622float2(h);
  }
  static __device__ __forceinline__ uint32_t from_f2(float2 f) {
    __nv_bfloat162 h = __float22bfloat162_rn(f);
    return *reinterpret_cast<uint32_t*>(&h);
  }
  static __device__ __forceinline__ uint16_t from_f(float f) { return __bfloat16_as_ushort(__float2bfloat16_rn(f)); }
};

// FP32 x-pairs: two FP32 values in one 8-byte word (deviations, unscaled).
template <> struct Pack2<Store::F32> {
  static __device__ __forceinline__ float2 to_f2(uint2 b) { return make_float2(__uint_as_float(b.x), __uint_as_float(b.y)); }
  static __device__ __forceinline__ uint2 from_f2(float2 f) { return make_uint2(__float_as_uint(f.x), __float_as_uint(f.y)); }
};

// An x-pair's storage word (lo = cell x0, hi = cell x0 + 1): two 16-bit
// values in 32 bits (FP16, BF16) or two FP32 values in 64 bits; H holds one
// value's bits.
template <Store S> struct PairWord { using W = uint32_t; using H = uint16_t; };
template <> struct PairWord<Store::F32> { using W = uint2; using H = uint32_t; };
__device__ __forceinline__ uint32_t lo_of(uint32_t w) { return w & 0xffffu; }
__device__ __forceinline__ uint32_t hi_of(uint32_t w) { return w >> 16; }
__device__ __forceinline__ uint32_t lo_of(uint2 w) { return w.x; }
__device__ __forceinline__ uint32_t hi_of(uint2 w) { return w.y; }
template <class W> __device__ __forceinline__ W pair_make(uint32_t lo, uint32_t hi);
template <> __device__ __forceinline__ uint32_t pair_make<uint32_t>(uint32_t lo, uint32_t hi) {
  return (lo & 0xffffu) | (hi << 16);
}
template <> __device__ __forceinline__ uint2 pair_make<uint2>(uint32_t lo, uint32_t hi) { return make_uint2(lo, hi); }

// pair (lo = cell x0, hi = cell x0 + 1) from two 16-bit halves
__device__ __forceinline__ uint32_t pair_of(uint32_t lo16, uint32_t hi16) { return (lo16 & 0xffffu) | (hi16 << 16); }

// The pair kernels collide in stored units: one unit of the equilibrium
// bracket (3 p~ + e (3 + 4.5 e) - 1.5 u.u) of a population of weight class
// cls is eq_factor(cls) stored units -- unit for the 2-byte formats, which
// store d unit / w, and w itself for FP32, which stores d.
template <Store S>
__host__ __device__ constexpr float eq_factor(int cls) {
  return S == Store::F32 ? static_cast<float>(weight_of_class(cls)) : store_unit(S);
}

// Second half of a 2-byte x-pair update: decode the pulled pairs (boundary
// values already in place), moments, case rules, collision and the paired
// store.  Shared by the register-staged kernels and the shared-memory staged
// kernels, so both produce the same bits.
//
// The collision runs in the stored units g_q = d_q * unit / w_q (d_q the
// deviation f_q - 3 w_q p_shift), where the equilibrium needs no weight:
//   g_q' = (1 - omega) g_q + omega unit (3 p~ + e(3 + 4.5 e) - 1.5 u.u),
// e = c_q . u and p~ = sum d_q / 3 = p - p_shift, since the shift's own
// equilibrium cancels (sum w_q = 1, sum w_q c_q = 0).  The moments take
// d_q = g_q w_q / unit.  For the sphere channel the deviations are from the
// inflow's equilibrium (Encoding::br_ref): u gains u_ref, the collision
// subtracts omega unit br_ref[q] (Encoding::kref) and populations bounced off
// the solid (links0 / links1, bit q) are corrected.  live0 / live1: the cell is fluid (a solid
// cell's values are left as they are); store: write the moments.
//
// REC (2-byte cavity, staged kernels): an x-wall cell also writes its
// row's wall record (`rec_row`, WallRecord layout): the post-collision
// values the halfway bounce-back returns to it next step, 32 bytes per wall
// side in three aligned stores, so that the next step's tile finds them in
// one bulk copy instead of nine scattered rows.
template <Store S, CaseRule RULE, bool REC = false, bool SR = false, class P>
__device__ __forceinline__ void finish_pair_row(const StepArgs& a, const P& pl,
                                                const typename PairWord<S>::W (&raw)[Q], const int x0,
                                                const int j, const int k, const bool lid, const bool left_edge,
                                                const bool live0, const bool live1, const bool store,
                                                const uint32_t seed, const uint32_t links0 = 0,
                                                const uint32_t links1 = 0, uint16_t* rec_row = nullptr) {
  // -1.5 u.u below is formed two ways of the same value: the sphere's
  // staged kernels spill 24 bytes with one and none with the other
  constexpr bool NEGADD = RULE == CaseRule::SphereStd;
  float2 g[Q];
  float2 s = f2s(0.f), u = f2s(0.f), v = f2s(0.f), w = f2s(0.f);
  // the format's scales are compile-time values (store_scale; Encoding holds
  // the same numbers for the host and the other kernels)
  constexpr float UNIT = store_unit(S);
  static_assert(!REC || S != Store::F32, "wall records are for the 2-byte formats");
  static_assert(RULE != CaseRule::SphereStd || S != Store::F32, "the FP32 sphere runs the one-cell kernels");
  [[maybe_unused]] const float lid6 = static_cast<float>(6.0 * a.rho_w * a.lid_u);
  static_for<0, Q>([&](auto qc) {
    constexpr int q = decltype(qc)::value;
    constexpr int ex = D3Q27::ex[q], ey = D3Q27::ey[q], ez = D3Q27::ez[q];
    float2 x = Pack2<S>::to_f2(raw[q]);
    if constexpr (RULE == CaseRule::CavityStd && ex != 0 && ez < 0) {
      // moving lid: + 6 rho_w w_q (c_q . u_w), in stored units
      constexpr float FAC = eq_factor<S>(D3Q27::wclass[q]);
      const float lid_g = lid6 * FAC;
      if (lid) x = add2rn(x, f2s(ex > 0 ? lid_g : -lid_g));
    }
    if constexpr (RULE == CaseRule::SphereStd && ex > 0) {
      if (left_edge) x.x = a.enc.inlet_g[q];
    }
    // d_q = g_q w_q / unit enters each moment as one fused multiply-add
    constexpr float isc = static_cast<float>(1.0 / store_scale(S, D3Q27::wclass[q]));
    s = fma2rn(x, f2s(isc), s);
    if constexpr (ex != 0) u = fma2rn(x, f2s(ex > 0 ? isc : -isc), u);
    if constexpr (ey != 0) v = fma2rn(x, f2s(ey > 0 ? isc : -isc), v);
    if constexpr (ez != 0) w = fma2rn(x, f2s(ez > 0 ? isc : -isc), w);
    g[q] = x;
  });
  if constexpr (RULE == CaseRule::SphereStd) {
    if (links0 | links1) {
      // A population bounced off the solid came back as the cell's own
      // bb(q) value; against the inflow's equilibrium its deviation gains
      // unit (br_ref[bb(q)] - br_ref[q]) = -6 unit c_q.u_ref (e_x != 0
      // only), added here with its share of the moments.
      static_for<0, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        constexpr int ex = D3Q27::ex[q], ey = D3Q27::ey[q], ez = D3Q27::ez[q];
        if constexpr (ex != 0) {
          const float c = -6.f * static_cast<float>(ex) * a.enc.u_ref[0] * UNIT;
          const float2 dg = f2(((links0 >> q) & 1u) ? c : 0.f, ((links1 >> q) & 1u) ? c : 0.f);
          g[q] = add2rn(g[q], dg);
          constexpr float isc = static_cast<float>(1.0 / store_scale(S, D3Q27::wclass[q]));
          const float2 dd = mul2rn(dg, f2s(isc));
          s = add2rn(s, dd);
          u = ex > 0 ? add2rn(u, dd) : add2rn(u, f2(-dd.x, -dd.y));
          if constexpr (ey != 0) v = ey > 0 ? add2rn(v, dd) : add2rn(v, f2(-dd.x, -dd.y));
          if constexpr (ez != 0) w = ez > 0 ? add2rn(w, dd) : add2rn(w, f2(-dd.x, -dd.y));
        }
      });
    }
    // deviations are from the inflow's equilibrium: its velocity adds back
    u = add2rn(u, f2s(a.enc.u_ref[0]));
  }
  const int32_t b = a.base32 + k * a.sz32 + j * a.pitch32 + x0;
  const int64_t c0 = x0 + static_cast<int64_t>(a.nx) * (j + static_cast<int64_t>(a.ny) * k);
  float2 p = mul2rn(s, f2s(1.0f / 3.0f));
  case_rules<RULE>(a, x0, k, c0, u.x, v.x, w.x, p.x);
  case_rules<RULE>(a, x0 + 1, k, c0 + 1, u.y, v.y, w.y, p.y);
  if (store) {
    a.mu[c0] = live0 ? u.x : 0.f;
    a.mv[c0] = live0 ? v.x : 0.f;
    a.mw[c0] = live0 ? w.x : 0.f;
    a.mp[c0] = live0 ? static_cast<double>(p.x) + a.p_shift : a.p_shift;
    a.mu[c0 + 1] = live1 ? u.y : 0.f;
    a.mv[c0 + 1] = live1 ? v.y : 0.f;
    a.mw[c0 + 1] = live1 ? w.y : 0.f;
    a.mp[c0 + 1] = live1 ? static_cast<double>(p.y) + a.p_shift : a.p_shift;
  }
  const float om = static_cast<float>(a.omega);
  const float2 keep = f2s(1.0f - om);
  // -1.5 u.u, rounded as 1.5 u.u then negated
  const float2 uu = fma2rn(w, w, fma2rn(v, v, mul2rn(u, u)));
  float2 mudu15;
  if constexpr (NEGADD) {
    const float2 t15 = mul2rn(f2s(1.5f), uu);
    mudu15 = f2(-t15.x, -t15.y);
  } else {
    mudu15 = mul2rn(f2s(-1.5f), uu);
  }
  // omega eq_factor(cls) and omega eq_factor(cls) (3 p~ - 1.5 u.u), per
  // weight class (one value for the 2-byte formats, whose factor is the
  // same for every class)
  // FP32 relaxes its non-equilibrium part instead, g - omega (g - geq)
  // with geq = w (3 p~ + e (3 + 4.5 e) - 1.5 u.u) (K_c = w (3 p~ - 1.5 u.u)):
  // near tau = 1/2 (omega near 2) that form keeps FP32's rounding of g,
  // where (1 - omega) g + omega geq doubles it.
  constexpr int NCLS = S == Store::F32 ? 4 : 1;
  const float2 kb = fma2rn(p, f2s(3.0f), mudu15);
  float om_c[NCLS];
  float2 K_c[NCLS];
#pragma unroll
  for (int c = 0; c < NCLS; ++c) {
    om_c[c] = om * eq_factor<S>(c);
    K_c[c] = mul2rn(f2s(S == Store::F32 ? eq_factor<S>(c) : om_c[c]), kb);
  }
  // Collision and stores; a pair whose two cells are both updated (every
  // pair but those beside a solid or past the lattice's end) takes a copy of
  // the loop without the per-population choice between a paired and two
  // half stores.
  // Wall record (REC): the pair holds the x = 0 cell (lo) or the x = nx - 1
  // cell (hi; nx >= 4, so not both).  Slot m of a side holds the 16-bit
  // value of pair m's population that leaves the box through that wall:
  // e_x = -1 (q = P_m + 1, low half of its word) at x = 0, e_x = +1 (q = P_m,
  // high half) at x = nx - 1; each is stored as the loop produces it, after
  // the side's zero padding (slots 9-15).
  [[maybe_unused]] const bool rec_lo = REC && x0 == 0, rec_hi = REC && x0 + 2 >= a.nx;
  if constexpr (REC) {
    if (rec_lo || rec_hi)
      *reinterpret_cast<uint4*>(rec_row + (rec_hi ? WallRecord::HI : 0) + 8) = make_uint4(0u, 0u, 0u, 0u);
  }
  // SR: stochastic rounding, the pair's random bits from x
  [[maybe_unused]] const uint32_t x = SR ? sr_hash(static_cast<uint32_t>(c0) ^ seed) : 0u;
  auto collide_store = [&](auto both_c) __attribute__((always_inline)) {
    constexpr bool BOTH = decltype(both_c)::value;
    static_for<0, Q>([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      constexpr int ci = NCLS == 1 ? 0 : D3Q27::wclass[q];
      [[maybe_unused]] const float om_u = om_c[ci];  // the 2-byte formats' collision
      const float2 K = K_c[ci];
      [[maybe_unused]] float2 Kq = K;
      if constexpr (RULE == CaseRule::SphereStd) {
        // minus the reference flow's equilibrium, omega unit br_ref[q]
        Kq = add2rn(K, f2s(a.enc.kref[q]));
      }
      const float2 gq = g[q];
      float2 gn;
      if constexpr (S == Store::F32) {
        constexpr float W = eq_factor<S>(D3Q27::wclass[q]);
        float2 geq = K;
        if constexpr (q != 0) {
          const float2 e = edu2<q>(u, v, w);
          geq = fma2rn(e, fma2rn(e, f2s(4.5f * W), f2s(3.0f * W)), K);
        }
        gn = fma2rn(f2s(-om), sub2rn(gq, geq), gq);
      } else if constexpr (q == 0) {
        gn = fma2rn(gq, keep, Kq);
      } else {
        // with e negated, so are the factors 4.5 and omega unit: same values.
        // The sphere's kernels keep the signed e, whose negations cost no
        // register for -omega unit (their registers are at the limit).
        constexpr bool en = RULE != CaseRule::SphereStd && edu_neg<q>();
        const float2 e = RULE != CaseRule::SphereStd ? edu2f<q>(u, v, w) : edu2<q>(u, v, w);
        const float2 t = fma2rn(e, f2s(en ? -4.5f : 4.5f), f2s(3.0f));
        const float2 h = mul2rn(e, f2s(en ? -om_u : om_u));
        gn = fma2rn(h, t, fma2rn(gq, keep, Kq));
      }
      typename PairWord<S>::W word;
      if constexpr (SR)
        word = sr_pair<S>(gn, x * sr_mul(q));
      else
        word = Pack2<S>::from_f2(gn);
      if constexpr (BOTH) {
        pl.store_pair(q, b, word);
        if constexpr (REC) {
          constexpr int ex = D3Q27::ex[q];
          if constexpr (ex < 0) {
            if (rec_lo) rec_row[WallRecord::slot(q)] = static_cast<uint16_t>(word & 0xffffu);
          } else if constexpr (ex > 0) {
            if (rec_hi) rec_row[WallRecord::HI + WallRecord::slot(q)] = static_cast<uint16_t>(word >> 16);
          }
        }
      } else {
        using H = typename PairWord<S>::H;
        if (live0) pl.store_half(q, b, static_cast<H>(lo_of(word)));
        if (live1) pl.store_half(q, b + 1, static_cast<H>(hi_of(word)));
      }
    });
  };
  if (live0 && live1)
    collide_store(std::true_type{});
  else
    collide_store(std::false_type{});
}

template <Store S, Bc B, CaseRule RULE, bool SR = false, class P>
__device__ __forceinline__ void step_cells_x2(const StepArgs& a, const P& pl, const int x0, const int j0, const int k) {
  constexpr int RY = PairRows<S>::value;
  using W = typename PairWord<S>::W;
  const bool xin = x0 < a.nx;  // nx even: both cells of the pair or neither
  const int xs = xin ? x0 : a.nx - 2;
  const bool left_edge = xs == 0, right_edge = xs + 2 >= a.nx;
  W raw[RY][Q];
  int32_t rowb[RY][3][3];  // [r][1 - ez][1 - ey]: index of x = xs in the source row
  bool act[RY];
  uint32_t row_out_bits[RY];  // cavity: bit (3 dz + dy) = source row outside the box
  uint32_t lid_mask = 0;      // cavity: rows whose cells sit under the lid
  uint32_t lk[RY][2];         // sphere: per-cell solid-link bits
  int32_t bself[RY];

  // Every population of both rows arrives as aligned 4-byte pairs issued
  // back to back.  A population with e_x = +1 needs (x0 - 1, x0): the high
  // half of the pair at x0 - 2 and the low half of the pair at x0; e_x = -1
  // needs (x0 + 1, x0 + 2) from the pairs at x0 and x0 + 2.  The second pair
  // is the neighbouring thread's own pair, so it shares the warp's cache
  // lines.  At the ends of a row the second pair's address carries the x
  // rule: the periodic image, or any in-range pair whose value a wall or the
  // inlet then replaces.
#pragma unroll
  for (int r = 0; r < RY; ++r) {
    const int j = j0 + r;
    act[r] = xin && j < a.ny;
    const int js = j < a.ny ? j : a.ny - 1;
    const int32_t b = a.base32 + k * a.sz32 + js * a.pitch32 + xs;  // own pair, aligned
    bself[r] = b;
    row_out_bits[r] = 0;
    if constexpr (B == Bc::Ghost) {
#pragma unroll
      for (int dz = 0; dz < 3; ++dz)
#pragma unroll
        for (int dy = 0; dy < 3; ++dy) rowb[r][dz][dy] = b - (1 - dz) * a.sz32 - (1 - dy) * a.pitch32;
    } else {
      const bool wrap = B == Bc::Periodic || RULE == CaseRule::SphereStd;
      const int jj[3] = {js == 0 ? (wrap ? a.ny - 1 : -1) : js - 1, js, js == a.ny - 1 ? (wrap ? 0 : a.ny) : js + 1};
      const int kk[3] = {k == 0 ? (wrap ? a.nz - 1 : -1) : k - 1, k, k == a.nz - 1 ? (wrap ? 0 : a.nz) : k + 1};
#pragma unroll
      for (int dz = 0; dz < 3; ++dz)
#pragma unroll
        for (int dy = 0; dy < 3; ++dy) {
          const bool out = jj[dy] < 0 || jj[dy] >= a.ny || kk[dz] < 0 || kk[dz] >= a.nz;
          if (out) row_out_bits[r] |= 1u << (3 * dz + dy);
          rowb[r][dz][dy] = out ? b : a.base32 + kk[dz] * a.sz32 + jj[dy] * a.pitch32 + xs;
        }
    }
    uint32_t links0 = 0, links1 = 0;
    if constexpr (RULE == CaseRule::SphereStd) {
      const bool near = act[r] && k >= a.near_lo[2] && k <= a.near_hi[2] && js >= a.near_lo[1] &&
                        js <= a.near_hi[1] && xs + 1 >= a.near_lo[0] && xs <= a.near_hi[0];
      const int64_t cell = xs + static_cast<int64_t>(a.nx) * (js + static_cast<int64_t>(a.ny) * k);
      links0 = near ? a.links[cell] : 0u;
      links1 = near ? a.links[cell + 1] : 0u;
    }
    lk[r][0] = links0;
    lk[r][1] = links1;
    if constexpr (RULE == CaseRule::CavityStd) {
      if (k == a.nz - 1) lid_mask |= 1u << r;
    }
    // offset of the neighbouring pair on each side, x rule included
    int32_t dleft, dright;
    if constexpr (B == Bc::Periodic) {
      dleft = left_edge ? a.nx - 2 : -2;
      dright = right_edge ? 2 - a.nx : 2;
    } else if constexpr (B == Bc::Ghost) {
      dleft = -2;
      dright = 2;
    } else {
      dleft = left_edge ? 0 : -2;   // wall / inlet replace the value
      dright = right_edge ? 0 : 2;  // wall replaces it; the outlet keeps the own column
    }
    static_for<0, Q>([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      constexpr int ex = D3Q27::ex[q], ey = D3Q27::ey[q], ez = D3Q27::ez[q];
      [[maybe_unused]] constexpr int qb = D3Q27::bb[q];
      const int32_t srow = rowb[r][1 - ez][1 - ey];
      const W pv = pl.load_pair(q, srow);
      W v = pv;
      if constexpr (ex == 1) {
        const W lv = pl.load_pair(q, srow + dleft);
        v = pair_make<W>(hi_of(lv), lo_of(pv));
      } else if constexpr (ex == -1) {
        const W rv = pl.load_pair(q, srow + dright);
        uint32_t rlo = lo_of(rv);
        if constexpr (RULE == CaseRule::SphereStd) {
          if (right_edge) rlo = hi_of(pv);  // zero-gradient outlet: the own column
        }
        v = pair_make<W>(hi_of(pv), rlo);
      }
      if constexpr (RULE == CaseRule::CavityStd) {
        // halfway bounce-back: a link leaving the box returns the cell's own
        // opposite population
        const bool out_row = (row_out_bits[r] >> (3 * (1 - ez) + (1 - ey))) & 1u;
        const bool out0 = out_row || (ex == 1 && left_edge);
        const bool out1 = out_row || (ex == -1 && right_edge);
        // a predicated load, not a branch: the x-wall lanes of a warp load
        // while the others do not, and no warp splits
        const W bbp = (out0 || out1) ? pl.load_pair(qb, b) : v;
        v = pair_make<W>(out0 ? lo_of(bbp) : lo_of(v), out1 ? hi_of(bbp) : hi_of(v));
      } else if constexpr (RULE == CaseRule::SphereStd) {
        const bool s0 = (links0 >> q) & 1u, s1 = (links1 >> q) & 1u;
        if (s0 || s1) {
          const W bbp = pl.load_pair(qb, b);
          v = pair_make<W>(s0 ? lo_of(bbp) : lo_of(v), s1 ? hi_of(bbp) : hi_of(v));
        }
      }
      raw[r][q] = v;
    });
  }

#pragma unroll
  for (int r = 0; r < RY; ++r) {
    if (!act[r]) continue;
    bool live0 = true, live1 = true;  // sphere: fluid cells (solid cells keep their values)
    if constexpr (RULE == CaseRule::SphereStd) {
      const int64_t c0 = x0 + static_cast<int64_t>(a.nx) * (j0 + r + static_cast<int64_t>(a.ny) * k);
      live0 = a.usr[c0] != 0;
      live1 = a.usr[c0 + 1] != 0;
    }
    finish_pair_row<S, RULE, false, SR>(a, pl, raw[r], x0, j0 + r, k, (lid_mask >> r) & 1u, left_edge, live0, live1,
                                        a.store, a.seed, lk[r][0], lk[r][1]);
  }
}

}  // namespace core
}  // namespace imx
