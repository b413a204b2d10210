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
#include <math_constants.h>

#include <type_traits>
#include <utility>

#include "lattice.h"
#include "step_core.cuh"
#include "stage_core.cuh"

namespace imx {
namespace {

constexpr int RED_THREADS_DRAG = 256;

// the per-cell machinery lives in step_core.cuh (shared with engine.cu)
using namespace core;

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
    [[maybe_unused]] constexpr int cls = D3Q27::wclass[q];
    R fq = feq_of<q, R, EXACT>(uu, vv, ww, tp3, udu15);
    if constexpr (S == Store::F16 || S == Store::BF16)
      fq -= wgt<R>(cls) * R(enc.br_ref[q]);  // deviation from the reference flow (0 unless set)
    const auto val = encode<S>(fq, q, enc);
    b0[b + q * L.sq] = val;
    if (b1) b1[b + q * L.sq] = val;
  });
}

// Initial fields of the standard sphere channel over the interior (x
// fastest): the inflow velocity (ui, 0, 0) in the fluid, rest in the solid,
// zero pressure deviation; out holds u, then v, w, p (n values each).
__global__ void sphere_fields_kernel(const uint8_t* fluid, int64_t n, double ui, double* out) {
  for (int64_t c = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; c < n;
       c += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    out[c] = fluid[c] ? ui : 0.0;
    out[n + c] = 0.0;
    out[2 * n + c] = 0.0;
    out[3 * n + c] = 0.0;
  }
}

// Programmatic dependent launch of consecutive steps (launch_pdl): a step
// kernel may be scheduled while the previous one drains; pdl_wait holds it,
// before its first access to global memory, until the previous grid has
// completed and its writes are visible, and pdl_release lets the next one
// be scheduled.  Both are no-ops for a kernel launched without the attribute.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <Store S, Bc B, CaseRule RULE, bool EXACT, bool DRAG>
__global__ void __launch_bounds__(256, 2) step_kernel(const StepArgs a) {
  pdl_release();
  pdl_wait();
  using T = typename StoreT<S>::T;
  constexpr int CPT = CellsPerThread<S>::value;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j0 = (blockIdx.y * blockDim.y + threadIdx.y) * CPT;
  int k = blockIdx.z;
  double drag[3] = {0.0, 0.0, 0.0};
  const Planes<T> pl{reinterpret_cast<const T* const*>(a.srcq), reinterpret_cast<T* const*>(a.dstq)};
  if constexpr (RULE == CaseRule::CavityRef) {
    // reference cavity with per-link boundaries: the first face_layers
    // z-layers of blocks take the face cells, one a thread, from the face
    // list (scheduled first, they run alongside the inside blocks)
    if (k < a.face_layers) {
      const int64_t e = ((static_cast<int64_t>(k) * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x) *
                            (blockDim.x * blockDim.y) +
                        threadIdx.y * blockDim.x + threadIdx.x;
      if (e < a.n_face) {
        const int32_t c = a.face_cells[e];
        const int fi = c % a.nx, fj = (c / a.nx) % a.ny, fk = c / (a.nx * a.ny);
        typename StoreT<S>::R f[Q];
        load_cell<S, B, RULE, EXACT, DRAG>(a, pl, fi, fj, fk, f, drag);
        compute_cell<S, RULE, EXACT>(a, pl, fi, fj, fk, f);
      }
      return;
    }
    k -= a.face_layers;
  }
  step_cells<S, B, RULE, EXACT, DRAG>(a, pl, i, j0, k, drag);

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

// 2-byte formats with nx even: each thread owns an x-pair in two rows
// (step_cells_x2); blockDim.x threads along x cover 2 blockDim.x cells.
// FP32 vortex and standard cavity with nx even: x-pairs of one row.
template <Store S, Bc B, CaseRule RULE, bool SR>
__global__ void __launch_bounds__(256, 2) step_kernel_x2(const StepArgs a) {
  pdl_release();
  pdl_wait();
  using T = typename StoreT<S>::T;
  const int x0 = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  const int j0 = PairRows<S>::value * (blockIdx.y * blockDim.y + threadIdx.y);
  const int k = blockIdx.z;
  const Planes<T> pl{reinterpret_cast<const T* const*>(a.srcq), reinterpret_cast<T* const*>(a.dstq)};
  step_cells_x2<S, B, RULE, SR>(a, pl, x0, j0, k);
}

// 2-byte formats, standard and periodic boundaries: rows staged in shared
// memory by bulk copies (stage_core.cuh).  A persistent grid; block b takes
// tiles b, b + grid, ... (y fastest, then z), so the blocks in flight cover
// a few consecutive planes.  Warp 0 also issues the copies.
template <Store S, Bc B, CaseRule RULE, bool SR>
__global__ void __launch_bounds__(stage::THREADS, 2) staged_kernel(const StepArgs a, const stage::Geo g) {
  using T = typename StoreT<S>::T;
  using namespace stage;
  constexpr bool WRAP = B == Bc::Periodic || RULE == CaseRule::SphereStd;
  constexpr bool REC = RULE == CaseRule::CavityStd;  // wall records staged with the rows
  extern __shared__ __align__(128) unsigned char smem[];
  T* stages = reinterpret_cast<T*>(smem);
  unsigned char* recs = smem + static_cast<size_t>(Q) * SLOT_UNITS * sizeof(T);
  uint64_t* full = reinterpret_cast<uint64_t*>(recs + (REC ? MAX_STAGES * REC_STAGE_BYTES : 0));
  uint64_t* empty = full + MAX_STAGES;
  auto rec_stage = [&](int sn) { return reinterpret_cast<uint16_t*>(recs + sn * REC_STAGE_BYTES); };
  __shared__ int abort_flag;
  constexpr int NS = MAX_STAGES;
  constexpr int stage_elems = Q * SLOT_CAP;
  if (threadIdx.x == 0) {
    for (int s = 0; s < NS; ++s) {
      bar_init(&full[s], 1);
      bar_init(&empty[s], THREADS / 32);
    }
    abort_flag = 0;
    bar_init_fence();
  }
  pdl_release();
  pdl_wait();  // the barriers above are set up while the previous step drains
  __syncthreads();
  volatile int* abort_v = &abort_flag;
  const int ntiles = g.nty * a.nz;
  const int grid = gridDim.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const T* src = static_cast<const T*>(a.src);
  // the sphere's linked pairs also load from global memory; its kernels keep
  // the per-population plane table (with strided planes they spill)
  using PL = std::conditional_t<RULE == CaseRule::SphereStd, Planes<T>, StridedPlanes<T>>;
  PL pl;
  if constexpr (RULE == CaseRule::SphereStd)
    pl = PL{reinterpret_cast<const T* const*>(a.srcq), reinterpret_cast<T* const*>(a.dstq)};
  else
    pl = PL{src, static_cast<T*>(a.dst), a.sq};

  // the block's first NS - 1 tiles
  int issued = 0;  // tiles of this block whose copies are issued (warp 0)
  if (warp == 0) {
    for (; issued < NS - 1; ++issued) {
      const int t = blockIdx.x + issued * grid;
      if (t >= ntiles) break;
      issue_tile<T, WRAP>(a, g, src, tile_origin(g, t), tile_plane(g, t), stages + issued * stage_elems, &full[issued],
                          REC ? a.rec_src : nullptr, rec_stage(issued));
    }
  }
  int i = 0;
  for (int t = blockIdx.x; t < ntiles; t += grid, ++i) {
    const int s = i % NS;
    if (warp == 0) {
      // refill the stage of tile i - 1 with tile i + NS - 1 once every warp
      // has released it; the decision to stop is warp-uniform
      const int tn = t + (NS - 1) * grid;
      if (tn < ntiles) {
        if (i > 0 && !__all_sync(0xffffffffu, bar_wait_for(&empty[(i - 1) % NS], ((i - 1) / NS) & 1u, a.wait_ns))) {
          *abort_v = 1;
          break;
        }
        const int sn = (i + NS - 1) % NS;
        issue_tile<T, WRAP>(a, g, src, tile_origin(g, tn), tile_plane(g, tn), stages + sn * stage_elems, &full[sn],
                            REC ? a.rec_src : nullptr, rec_stage(sn));
        ++issued;
      }
    }
    if (!__all_sync(0xffffffffu, bar_wait_for(&full[s], (i / NS) & 1u, a.wait_ns))) {
      *abort_v = 1;
      break;
    }
    const uint32_t* st = reinterpret_cast<const uint32_t*>(stages + s * stage_elems);
    consume_tile<S, B, RULE, SR>(a, pl, g, st, tile_origin(g, t), tile_plane(g, t), a.store != 0, a.seed, rec_stage(s),
                             a.rec_dst);
    __syncwarp();
    if (lane == 0) bar_arrive(&empty[s]);
    if (__any_sync(0xffffffffu, *abort_v != 0)) break;
  }
  if (warp == 0 && lane == 0 && *abort_v) {
    // let copies still in flight land before the block exits (bounded by the
    // full second whatever a.wait_ns is)
    for (int m = i; m < issued; ++m) (void)bar_wait(&full[m % NS], (m / NS) & 1u);
  }
  __syncthreads();
  if (threadIdx.x == 0 && abort_flag) atomicOr(a.err, 1);
}

// 2-byte standard cavity: the wall records (WallRecord) of buffer `buf`,
// gathered from its x-wall cells: the state a step leaves them in, for the
// initial state and a loaded checkpoint.  One thread per row (j, k).
__global__ void cavity_records_kernel(const Layout L, const uint16_t* buf, uint16_t* rec) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y;
  if (j >= L.ny) return;
  uint32_t w[WallRecord::WORDS / 2] = {};
#pragma unroll
  for (int m = 0; m < WallRecord::SLOTS; ++m) {
    const int p = WallRecord::pos(m);
    const uint32_t lo = buf[L.idx(p + 1, 0, j, k)], hi = buf[L.idx(p, L.nx - 1, j, k)];
    w[m >> 1] |= lo << (16 * (m & 1));
    w[(WallRecord::HI + m) >> 1] |= hi << (16 * (m & 1));
  }
  uint4* out = reinterpret_cast<uint4*>(rec + (static_cast<int64_t>(k) * L.ny + j) * WallRecord::WORDS);
#pragma unroll
  for (int c = 0; c < 4; ++c) out[c] = make_uint4(w[4 * c], w[4 * c + 1], w[4 * c + 2], w[4 * c + 3]);
}

// Momentum-exchange drag of the 2-byte sphere channel, from the buffer a
// step reads: every fluid cell c with a solid link along -e_q takes back
// f*(bb(q), c), so the body receives -2 (f*(bb(q), c)) e_q.  Its own kernel
// over the box of linked cells, so the step kernels carry no drag code;
// per-block partial sums (3 per block) are added in a fixed order by
// drag_sum_kernel, so the force is deterministic.
template <Store S>
__global__ void __launch_bounds__(256) drag_links_kernel(const StepArgs a) {
  using T = typename StoreT<S>::T;
  const T* src = static_cast<const T*>(a.src);
  const int bx = a.near_hi[0] - a.near_lo[0] + 1, by = a.near_hi[1] - a.near_lo[1] + 1;
  const int bz = a.near_hi[2] - a.near_lo[2] + 1;
  const int64_t nbox = bx > 0 && by > 0 && bz > 0 ? static_cast<int64_t>(bx) * by * bz : 0;
  double acc[3] = {0.0, 0.0, 0.0};
  for (int64_t n = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; n < nbox;
       n += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int i = a.near_lo[0] + static_cast<int>(n % bx);
    const int j = a.near_lo[1] + static_cast<int>((n / bx) % by);
    const int k = a.near_lo[2] + static_cast<int>(n / (static_cast<int64_t>(bx) * by));
    const int64_t cell = i + static_cast<int64_t>(a.nx) * (j + static_cast<int64_t>(a.ny) * k);
    const uint32_t bits = a.links[cell];
    if (!bits) continue;
    const int64_t b = a.base + k * a.sz + j * a.pitch + i;
    static_for<0, Q>([&](auto qc) {
      constexpr int q = decltype(qc)::value;
      constexpr int qb = D3Q27::bb[q], cls = D3Q27::wclass[q];
      constexpr int ex = D3Q27::ex[q], ey = D3Q27::ey[q], ez = D3Q27::ez[q];
      if ((bits >> q) & 1u) {
        const T raw = src[static_cast<int64_t>(qb) * a.sq + b];
        float d;
        if constexpr (S == Store::F16) d = __fmul_rn(__half2float(raw), a.enc.inv_scale[qb]);
        else d = __fmul_rn(__bfloat162float(raw), a.enc.inv_scale[qb]);
        const double f = static_cast<double>(d) +
                         wgt<double>(cls) * (3.0 * a.p_shift + static_cast<double>(a.enc.br_ref[qb]));
        if constexpr (ex != 0) acc[0] -= 2.0 * f * ex;
        if constexpr (ey != 0) acc[1] -= 2.0 * f * ey;
        if constexpr (ez != 0) acc[2] -= 2.0 * f * ez;
      }
    });
  }
  __shared__ double sh[3][8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    double x = acc[c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) sh[c][warp] = x;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double x = 0.0;
    for (int w = 0; w < 8; ++w) x += sh[threadIdx.x][w];
    a.drag_part[3 * blockIdx.x + threadIdx.x] = x;
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
  // Four independent entries per thread with every load issued before any
  // store: the gather is latency-bound (each entry is an index load followed
  // by a dependent value load), so independent entries in flight are what
  // sets its speed.  Targets never alias this step's sources (the plan is
  // refused otherwise), so the order of the copies does not matter.
  using T = typename StoreT<S>::T;
  constexpr int V = 4;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x * V;
  for (int64_t e0 = static_cast<int64_t>(blockIdx.x) * blockDim.x * V + threadIdx.x; e0 < n; e0 += stride) {
    int64_t s[V], t[V];
#pragma unroll
    for (int u = 0; u < V; ++u) {
      const int64_t e = e0 + static_cast<int64_t>(u) * blockDim.x;
      s[u] = e < n ? src[e] : -1;
      t[u] = e < n ? tgt[e] : -1;
    }
    T val[V];
#pragma unroll
    for (int u = 0; u < V; ++u) {
      if (s[u] >= 0) {
        val[u] = dst[s[u]];
      } else if (s[u] <= -2) {
        val[u] = prev[-s[u] - 2];
      } else {
        val[u] = encode<S>(typename StoreT<S>::R(0), t[u] >= 0 ? static_cast<int>(t[u] / sq) : 0, enc);
      }
    }
#pragma unroll
    for (int u = 0; u < V; ++u)
      if (t[u] >= 0) dst[t[u]] = val[u];
  }
}

// The same gather over a packed plan: entry e is (target, source) as two
// 32-bit indices (int2), one 8-byte load instead of two.  Launched with
// programmatic dependent launch after the step kernel: the plan does not
// depend on the step, so a thread loads its first entries while the step
// kernel drains and only then waits for the step's values (pdl_wait).
template <Store S>
__global__ void ghost_gather_packed_kernel(typename StoreT<S>::T* __restrict__ dst,
                                           const typename StoreT<S>::T* __restrict__ prev,
                                           const int2* __restrict__ plan, int64_t n, int64_t sq, Encoding enc) {
  using T = typename StoreT<S>::T;
  constexpr int V = 4;
  pdl_release();
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x * V;
  int64_t e0 = static_cast<int64_t>(blockIdx.x) * blockDim.x * V + threadIdx.x;
  int2 p[V];
  auto load_plan = [&]() {
#pragma unroll
    for (int u = 0; u < V; ++u) {
      const int64_t e = e0 + static_cast<int64_t>(u) * blockDim.x;
      p[u] = e < n ? __ldg(plan + e) : make_int2(-1, -1);
    }
  };
  load_plan();
  pdl_wait();  // the step kernel's values are complete and visible from here on
  for (; e0 < n; e0 += stride) {
    T val[V];
#pragma unroll
    for (int u = 0; u < V; ++u) {
      if (p[u].y >= 0) {
        val[u] = dst[p[u].y];
      } else if (p[u].y <= -2) {
        val[u] = prev[-static_cast<int64_t>(p[u].y) - 2];
      } else {
        val[u] = encode<S>(typename StoreT<S>::R(0), p[u].x >= 0 ? static_cast<int>(p[u].x / sq) : 0, enc);
      }
    }
#pragma unroll
    for (int u = 0; u < V; ++u)
      if (p[u].x >= 0) dst[p[u].x] = val[u];
    if (e0 + stride < n) {
      e0 += stride;
      load_plan();
      e0 -= stride;
    }
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

// Both sums of the velocity residual in one pass over (u, v, w) and the
// previous (u2, v2, w2): part[2 b] = sum |u - u2|^2, part[2 b + 1] = sum |u|^2
// over block b's slice (the same slices and order as reduce_pass1), then
// one block adds the partials in order into out[0], out[1].
__global__ void resid_pass1(const double* u, const double* v, const double* w, const double* u2, const double* v2,
                            const double* w2, int64_t n, double* part) {
  double d2 = 0.0, n2 = 0.0;
  for (int64_t c = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; c < n;
       c += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double a = u[c], b = v[c], g = w[c];
    const double du = a - u2[c], dv = b - v2[c], dw = g - w2[c];
    d2 += du * du + dv * dv + dw * dw;
    n2 += a * a + b * b + g * g;
  }
  __shared__ double sh[2][RED_THREADS / 32];
  d2 = warp_sum(d2);
  n2 = warp_sum(n2);
  if ((threadIdx.x & 31) == 0) {
    sh[0][threadIdx.x >> 5] = d2;
    sh[1][threadIdx.x >> 5] = n2;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    double x = threadIdx.x < RED_THREADS / 32 ? sh[0][threadIdx.x] : 0.0;
    double y = threadIdx.x < RED_THREADS / 32 ? sh[1][threadIdx.x] : 0.0;
    x = warp_sum(x);
    y = warp_sum(y);
    if (threadIdx.x == 0) {
      part[2 * blockIdx.x] = x;
      part[2 * blockIdx.x + 1] = y;
    }
  }
}

__global__ void resid_pass2(const double* part, int nparts, double* out) {
  double x = 0.0, y = 0.0;
  for (int c = threadIdx.x; c < nparts; c += blockDim.x) {
    x += part[2 * c];
    y += part[2 * c + 1];
  }
  __shared__ double sh[2][RED_THREADS / 32];
  x = warp_sum(x);
  y = warp_sum(y);
  if ((threadIdx.x & 31) == 0) {
    sh[0][threadIdx.x >> 5] = x;
    sh[1][threadIdx.x >> 5] = y;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    double a = threadIdx.x < RED_THREADS / 32 ? sh[0][threadIdx.x] : 0.0;
    double b = threadIdx.x < RED_THREADS / 32 ? sh[1][threadIdx.x] : 0.0;
    a = warp_sum(a);
    b = warp_sum(b);
    if (threadIdx.x == 0) {
      out[0] = a;
      out[1] = b;
    }
  }
}

// The velocity residual sqrt(num / den) from the two sums of the residual
// reduction, as the synchronous path forms it on the host (INFINITY on the
// first call, NaN when a sum is not finite).
__global__ void residual_finish_kernel(const double* nd, int first, double* out) {
  const double num = nd[0], den = nd[1];
  double r;
  if (first)
    r = CUDART_INF;
  else if (!isfinite(num) || !isfinite(den))
    r = CUDART_NAN;
  else
    r = den > 0.0 ? sqrt(num / den) : (num > 0.0 ? CUDART_INF : 0.0);
  *out = r;
}

}  // namespace

cudaError_t launch_residual_sums(const double* u, const double* v, const double* w, const double* u2,
                                 const double* v2, const double* w2, int64_t n, double* scratch, double* out,
                                 cudaStream_t s) {
  resid_pass1<<<RED_BLOCKS, RED_THREADS, 0, s>>>(u, v, w, u2, v2, w2, n, scratch);
  resid_pass2<<<1, RED_THREADS, 0, s>>>(scratch, RED_BLOCKS, out);
  return cudaGetLastError();
}

cudaError_t launch_residual_finish(const double* nd, int first, double* out, cudaStream_t s) {
  residual_finish_kernel<<<1, 1, 0, s>>>(nd, first, out);
  return cudaGetLastError();
}

dim3 step_block(int nx) {
  if (nx >= 128) return dim3(128, 2, 1);
  if (nx >= 64) return dim3(64, 4, 1);
  return dim3(32, 8, 1);
}

// 2-byte x-pair kernel: threads along x cover two cells each
static dim3 step_block_x2(int nx) {
  if (nx >= 128) return dim3(64, 4, 1);
  if (nx >= 64) return dim3(32, 8, 1);
  return dim3(16, 16, 1);
}

static bool use_x2(Store s, int nx) { return (s == Store::F16 || s == Store::BF16) && nx % 2 == 0; }

// Shared-memory staged kernel: 2-byte formats with nx even and the standard
// or periodic boundaries, rows of at most 1024 stored elements.
static bool staged_geo(const LaunchCfg& c, int nx, int ny, int64_t pitch, stage::Geo* g) {
  if (!use_x2(c.store, nx)) return false;
  if (c.bc != Bc::Standard && c.bc != Bc::Periodic) return false;
  return stage::staged_layout(c.rule, nx, ny, pitch, g);
}

bool uses_wall_records(const LaunchCfg& c, int nx, int ny, int64_t pitch) {
  stage::Geo g;
  return c.rule == CaseRule::CavityStd && staged_geo(c, nx, ny, pitch, &g);
}

// Blocks of the persistent staged grid: as many as fit on the device at
// once (queried once per kernel), no more than there are tiles.
static int device_sms() {
  static int sms = 0;
  if (sms == 0) {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    sms = n > 0 ? n : 148;
  }
  return sms;
}

template <Store S, Bc B, CaseRule R, bool SR>
static int staged_blocks(const stage::Geo& g, int nz) {
  static int resident = 0;  // blocks of this kernel resident on the device
  if (resident == 0) {
    const size_t smem = stage::smem_bytes(static_cast<int>(sizeof(typename StoreT<S>::T)), R == CaseRule::CavityStd);
    cudaFuncSetAttribute(staged_kernel<S, B, R, SR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(smem));
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, staged_kernel<S, B, R, SR>, stage::THREADS, smem);
    resident = (per_sm > 0 ? per_sm : 1) * device_sms();
  }
  const int64_t ntiles = static_cast<int64_t>(g.nty) * nz;
  return static_cast<int>(ntiles < resident ? ntiles : resident);
}

template <Store S, Bc B, CaseRule R, bool SR>
static cudaError_t launch_staged(const StepArgs& a, const stage::Geo& g, cudaStream_t s) {
  const size_t smem = stage::smem_bytes(static_cast<int>(sizeof(typename StoreT<S>::T)), R == CaseRule::CavityStd);
  if (R == CaseRule::CavityStd && (!a.rec_src || !a.rec_dst)) return cudaErrorInvalidValue;
  const int blocks = staged_blocks<S, B, R, SR>(g, a.nz);
  return launch_pdl(staged_kernel<S, B, R, SR>, dim3(blocks), dim3(stage::THREADS), smem, s, a, g);
}

// ------------------------------------------------------------ launchers
int reduce_blocks() { return RED_BLOCKS; }

constexpr int DRAG_LINK_BLOCKS = 148;

bool drag_in_own_kernel(Store s) { return s == Store::F16 || s == Store::BF16; }

cudaError_t launch_drag_links(Store st, const StepArgs& a, cudaStream_t s) {
  if (st == Store::F16)
    drag_links_kernel<Store::F16><<<DRAG_LINK_BLOCKS, 256, 0, s>>>(a);
  else if (st == Store::BF16)
    drag_links_kernel<Store::BF16><<<DRAG_LINK_BLOCKS, 256, 0, s>>>(a);
  else
    return cudaErrorInvalidValue;
  return cudaGetLastError();
}

int64_t step_grid_blocks(const LaunchCfg& c, int nx, int ny, int nz) {
  if (drag_in_own_kernel(c.store)) return DRAG_LINK_BLOCKS;
  const dim3 b = step_block(nx);
  const int cpt = c.store == Store::F64 ? 1 : CellsPerThread<Store::F32>::value;
  const int rows = b.y * cpt;
  return static_cast<int64_t>((nx + b.x - 1) / b.x) * ((ny + rows - 1) / rows) * nz;
}

// The staged kernels' copy plan of one 2-byte lattice, from the same
// tile_runs / tile_runs_flat the kernels run (see imexlb_debug_stage_plan).
int64_t stage_plan(int nx, int ny, int nz, int mode, int32_t* geo, int32_t* runs, int64_t max_runs) {
  const Layout L = make_layout(nx, ny, nz, 0, 2);
  stage::Geo g;
  const CaseRule rule = mode == 0 ? CaseRule::CavityStd : (mode == 2 ? CaseRule::SphereStd : CaseRule::None);
  if (!stage::staged_layout(rule, nx, ny, L.pitch, &g)) return -1;
  StepArgs a;
  a.nx = nx;
  a.ny = ny;
  a.nz = nz;
  a.base32 = static_cast<int32_t>(L.idx(0, 0, 0, 0));
  a.sz32 = static_cast<int32_t>(L.sz);
  a.pitch32 = static_cast<int32_t>(L.pitch);
  if (geo) {
    const int32_t v[10] = {g.P, g.R, g.cap, g.nty, static_cast<int32_t>(L.sq), a.sz32, a.pitch32, a.base32,
                           g.flat, g.C};
    for (int i = 0; i < 10; ++i) geo[i] = v[i];
  }
  int64_t n = 0;
  for (int t = 0; t < g.nty * nz; ++t) {
    const int j0 = stage::tile_origin(g, t), k = stage::tile_plane(g, t);
    const int rv = ny - j0 < g.R ? ny - j0 : g.R;
    for (int q = 0; q < Q; ++q) {
      stage::Run m{0, 0, 0u, q}, w{0, 0, 0u, q};
      if (g.flat)
        stage::tile_runs_flat(a, g, q, j0, k, 2, m, w);
      else if (rule != CaseRule::CavityStd)
        stage::tile_runs<true>(a, g, q, j0, k, rv, 2, m, w);
      else
        stage::tile_runs<false>(a, g, q, j0, k, rv, 2, m, w);
      for (const stage::Run* r : {&m, &w}) {
        if (!r->bytes) continue;
        if (runs && n < max_runs) {
          int32_t* o = runs + 6 * n;
          o[0] = t;
          o[1] = q;
          o[2] = r->pop;
          o[3] = r->src;
          o[4] = r->dst;
          o[5] = static_cast<int32_t>(r->bytes);
        }
        ++n;
      }
    }
    if (rule == CaseRule::CavityStd) {
      // the wall records: "population" Q, element offsets into the record
      // buffer and the stage's record area
      int64_t rsrc = 0;
      uint32_t rbytes = 0;
      stage::tile_records(a, j0, k, rv, rsrc, rbytes);
      if (runs && n < max_runs) {
        int32_t* o = runs + 6 * n;
        o[0] = t;
        o[1] = Q;
        o[2] = -1;
        o[3] = static_cast<int32_t>(rsrc);
        o[4] = 0;
        o[5] = static_cast<int32_t>(rbytes);
      }
      ++n;
    }
  }
  return n;
}

cudaError_t launch_cavity_records(const Layout& L, const void* buf, uint16_t* rec, cudaStream_t s) {
  if (L.elem != 2 || L.g != 0) return cudaErrorInvalidValue;
  const dim3 block(64, 1, 1), grid((L.ny + 63) / 64, L.nz, 1);
  cavity_records_kernel<<<grid, block, 0, s>>>(L, static_cast<const uint16_t*>(buf), rec);
  return cudaGetLastError();
}

cudaError_t launch_sphere_fields(const uint8_t* fluid, int64_t n, double ui, double* out, cudaStream_t s) {
  const int64_t want = (n + 255) / 256;
  sphere_fields_kernel<<<static_cast<int>(want < 148 * 16 ? want : 148 * 16), 256, 0, s>>>(fluid, n, ui, out);
  return cudaGetLastError();
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

// Launch with programmatic stream serialisation: the kernel may start
// while the kernel before it on the stream finishes (see pdl_wait).
template <class... KArgs, class... Args>
static cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                              Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// SR: the 2-byte pair kernels round their stores stochastically (Encoding::sr;
// the cavity and the sphere only)
template <Store S, Bc B, CaseRule R, bool EXACT, bool SR>
static cudaError_t step_pairs(const StepArgs& a, cudaStream_t s, bool* done) {
  *done = true;
  if constexpr (B == Bc::Standard || B == Bc::Periodic) {
    stage::Geo g;
    if (staged_geo(LaunchCfg{B, S, R, EXACT}, a.nx, a.ny, a.pitch, &g)) return launch_staged<S, B, R, SR>(a, g, s);
  }
  // (the 2-byte formats sum their drag in drag_links_kernel)
  if (use_x2(S, a.nx)) {
    const dim3 block = step_block_x2(a.nx);
    constexpr int RY = PairRows<S>::value;
    const dim3 grid((a.nx + 2 * block.x - 1) / (2 * block.x), (a.ny + RY * block.y - 1) / (RY * block.y), a.nz);
    return launch_pdl(step_kernel_x2<S, B, R, SR>, grid, block, 0, s, a);
  }
  *done = false;
  return cudaSuccess;
}

template <Store S, Bc B, CaseRule R, bool EXACT>
static cudaError_t step_impl(const StepArgs& a, cudaStream_t s) {
  if constexpr (S == Store::F32 && (R == CaseRule::None || R == CaseRule::CavityStd) &&
                (B == Bc::Standard || B == Bc::Periodic)) {
    if (a.nx % 2 == 0) {
      const dim3 block = step_block_x2(a.nx);
      const dim3 grid((a.nx + 2 * block.x - 1) / (2 * block.x), (a.ny + block.y - 1) / block.y, a.nz);
      return launch_pdl(step_kernel_x2<S, B, R, false>, grid, block, 0, s, a);
    }
  }
  if constexpr (S == Store::F16 || S == Store::BF16) {
    bool done = false;
    cudaError_t err;
    if constexpr (R == CaseRule::CavityStd || R == CaseRule::SphereStd)
      err = a.enc.sr ? step_pairs<S, B, R, EXACT, true>(a, s, &done) : step_pairs<S, B, R, EXACT, false>(a, s, &done);
    else
      err = step_pairs<S, B, R, EXACT, false>(a, s, &done);
    if (done) return err;
  }
  const dim3 block = step_block(a.nx);
  const int rows = block.y * CellsPerThread<S>::value;
  dim3 grid((a.nx + block.x - 1) / block.x, (a.ny + rows - 1) / rows, a.nz);
  if constexpr (R == CaseRule::CavityRef) {
    if (a.face_cells) {
      // the face blocks: leading z-layers of the grid, one face cell a thread
      StepArgs fa = a;
      const int64_t per_layer = static_cast<int64_t>(grid.x) * grid.y * block.x * block.y;
      fa.face_layers = static_cast<int32_t>((a.n_face + per_layer - 1) / per_layer);
      grid.z += fa.face_layers;
      return launch_pdl(step_kernel<S, B, R, EXACT, false>, grid, block, 0, s, fa);
    }
  }
  if constexpr (R == CaseRule::SphereStd && S != Store::F16 && S != Store::BF16) {
    if (a.drag_part) {
      return launch_pdl(step_kernel<S, B, R, EXACT, true>, grid, block, 0, s, a);
    }
  }
  return launch_pdl(step_kernel<S, B, R, EXACT, false>, grid, block, 0, s, a);
}

template <Store S, bool EXACT>
static cudaError_t step_rule(const LaunchCfg& c, const StepArgs& a, cudaStream_t s) {
  switch (c.rule) {
    case CaseRule::None: return step_impl<S, Bc::Periodic, CaseRule::None, EXACT>(a, s);
    case CaseRule::CavityRef: return step_impl<S, Bc::Ghost, CaseRule::CavityRef, EXACT>(a, s);
    case CaseRule::SphereRef: return step_impl<S, Bc::Ghost, CaseRule::SphereRef, EXACT>(a, s);
    case CaseRule::CavityStd: return step_impl<S, Bc::Standard, CaseRule::CavityStd, EXACT>(a, s);
    case CaseRule::SphereStd: return step_impl<S, Bc::Standard, CaseRule::SphereStd, EXACT>(a, s);
    case CaseRule::SlabStd:
      // FP64 and FP32 storage only (register kernels)
      if constexpr (S == Store::F64 || S == Store::F32)
        return step_impl<S, Bc::Standard, CaseRule::SlabStd, EXACT>(a, s);
      else
        return cudaErrorNotSupported;
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

cudaError_t launch_ghost_gather_packed(Store st, void* dst, const void* prev, const int2* plan, int64_t n, int64_t sq,
                                       const Encoding& enc, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const int threads = 256;
  const int64_t want = (n + threads * 4 - 1) / (threads * 4);
  const int blocks = static_cast<int>(want < 148 * 8 ? want : 148 * 8);
  cudaError_t err = cudaSuccess;
  switch (st) {
#define IMX_GGP(S)                                                                                               \
  case S:                                                                                                        \
    err = launch_pdl(ghost_gather_packed_kernel<S>, dim3(blocks), dim3(threads), 0, s,                         \
                     static_cast<typename StoreT<S>::T*>(dst), static_cast<const typename StoreT<S>::T*>(prev), \
                     plan, n, sq, enc);                                                                        \
    break;
    IMX_GGP(Store::F64)
    IMX_GGP(Store::F32)
    IMX_GGP(Store::F16)
    IMX_GGP(Store::BF16)
#undef IMX_GGP
  }
  return err != cudaSuccess ? err : cudaGetLastError();
}

cudaError_t launch_ghost_gather(Store st, void* dst, const void* prev, const int64_t* tgt, const int64_t* src,
                                int64_t n, int64_t sq, const Encoding& enc, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const int threads = 256;
  const int64_t want = (n + threads * 4 - 1) / (threads * 4);
  const int blocks = static_cast<int>(want < 148 * 8 ? want : 148 * 8);
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
