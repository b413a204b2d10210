// Engine: many independent lattices ("instances") of uneven sizes on one GPU,
// all advanced one time step per persistent kernel launch.
//
// Batched solves and the served request stream (no counterpart in the
// reference, which runs one lattice per process) need many small and medium
// lattices to share the GPU.  A launch per lattice per step would leave most
// of the 148 SMs idle on small lattices and pay a launch each; instead the
// engine keeps a device-side work list of (instance, tile) items covering
// every active instance, and one persistent launch per step walks it: block b
// takes items b, b + grid, b + 2 grid, ...  A tile is 256 threads' worth of
// cells of one instance (bx cells along x by 256/bx rows, times the cells per
// thread of the storage format); its tile width bx is chosen per instance
// (autotuned per size and storage).  A block copies the instance's arguments
// into shared memory once per change of instance and runs exactly the
// per-cell code of the single-lattice kernels (step_core.cuh).
//
// Instances live in one device arena reserved at creation: admission fails
// (IMEXLB_E_NOMEM) when an instance does not fit the arena's budget, which
// is how a server admits requests against an HBM budget.  Each instance keeps
// its own buffer parity, so instances join and leave between any two steps.
// Two consecutive steps are captured as a CUDA graph and replayed while the
// set of instances does not change.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/imexlb.h"
#include "lattice.h"
#include "step_core.cuh"
#include "stage_core.cuh"

namespace imx {
namespace {

using namespace core;

struct __align__(16) EngInst {
  StepArgs a;    // first member: the staged kernels copy its prefix from here
  void* buf[2];
  double* prev;  // u, v, w at the last residual check (3 n values)
  int rule;      // CaseRule
  int bx_log2;   // tile width 2^bx_log2 threads along x (register-staged kernels)
  int parity0;   // engine step parity at admission
  int x2;        // nx even, 2-byte format or FP32 vortex: threads own x-pairs (step_cells_x2)
  int staged;    // 2-byte format, rows staged in shared memory (stage_core.cuh)
  int tw, th;    // cells of a tile along x and y
  stage::Geo geo;
  uint16_t* rec[2];  // wall records of buf[0], buf[1] (staged 2-byte cavity), else null
};

struct Tile {
  int32_t slot, i0, j0, k;
};

// Everything warp 0 of a staged engine kernel needs to issue a tile's
// copies, flattened per tile (rebuild_tiles), 128 bytes: one word per lane,
// so the descriptor of the block's next tile arrives with one coalesced load
// while the current tile is computed.
struct __align__(128) StagedTile {
  const void* buf[2];     // distribution buffers of the instance
  uint16_t* rec[2];       // their wall records (staged cavity), else null
  const StepArgs* args;   // the instance's StepArgs (prefix copied per tile)
  int64_t sq;
  int32_t base32, sz32, pitch32;
  int nx, ny, nz;
  int parity0;
  int j0, k;
  stage::Geo geo;
  int slot;
};
static_assert(sizeof(StagedTile) == 128, "one 4-byte word per lane");

// 16 bytes from global to shared memory, asynchronously (cp.async; the
// issuing thread waits for its copies with cp_async_wait_all)
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(stage::smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

struct EngArgs {
  const EngInst* inst;
  const Tile* tiles;
  const StagedTile* stiles;  // staged groups: per-tile descriptors (index as tiles)
  const int* left;           // per slot: steps the instance still takes (ENG_NO_LIMIT: no limit)
  int ntiles;
  int parity;
  int store;
  int* err;  // set non-zero by a staged kernel that gave up waiting
  // per slot: steps the instance has taken (its stochastic-rounding seed is
  // the hash of this count, as for a single lattice)
  const uint32_t* seed = nullptr;
};

// What the consumer warps of a staged engine kernel need of a tile beyond
// its rows and its instance's StepArgs prefix: written to shared memory by
// warp 0 with the tile's copies (the stage's full mbarrier publishes it),
// so that no consumer waits on global loads of the tile list or instance.
struct __align__(16) TileHdr {
  const void* src;   // distribution buffer read
  void* dst;         // distribution buffer written
  uint16_t* rec;     // wall records written (staged cavity), else null
  stage::Geo geo;
  int j0, k;
  int skip;          // the instance has taken its steps: no copies, no update
  int store;         // write the moments (the call's last step or the instance's)
  uint32_t seed;     // the instance's stochastic-rounding seed for this step
};
constexpr size_t TILE_HDR_BYTES = (sizeof(TileHdr) + 15) & ~static_cast<size_t>(15);

// Steps left of an instance without a step limit (imexlb_engine_limit).
constexpr int ENG_NO_LIMIT = 0x7fffffff;

// Before each step a tile reads its instance's steps left: 0 skips the tile,
// 1 (the instance's last step) also writes the moments.  engine_tick counts
// them down after the step.
__global__ void engine_tick(int* left, uint32_t* taken, int n) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) {
    const int l = left[s];
    if (l > 0 && l != ENG_NO_LIMIT) left[s] = l - 1;
    if (l != 0) taken[s] += 1u;
  }
}

// Population planes of one instance: plane q starts q * sq elements into the
// buffer (27 sq < 2^31 for every engine instance).
template <class T>
struct FlatPlanes {
  const T* src;
  T* dst;
  int32_t sq;
  __device__ __forceinline__ T load(int q, int32_t idx) const { return ldg_stream(src + (q * sq + idx)); }
  __device__ __forceinline__ void store(int q, int32_t idx, T v) const { dst[q * sq + idx] = v; }
  // x-pair words: 32-bit pairs of 16-bit values; FP32: 64-bit pairs
  using W = std::conditional_t<sizeof(T) == 4, uint2, uint32_t>;
  using H = std::conditional_t<sizeof(T) == 4, uint32_t, uint16_t>;
  __device__ __forceinline__ W load_pair(int q, int32_t idx) const {
    return __ldg(reinterpret_cast<const W*>(src + (q * sq + idx)));
  }
  __device__ __forceinline__ uint32_t load_half(int q, int32_t idx) const {
    return __ldg(reinterpret_cast<const unsigned short*>(src + (q * sq + idx)));
  }
  __device__ __forceinline__ void store_pair(int q, int32_t idx, W v) const {
    *reinterpret_cast<W*>(dst + (q * sq + idx)) = v;
  }
  __device__ __forceinline__ void store_half(int q, int32_t idx, H v) const {
    *reinterpret_cast<H*>(dst + (q * sq + idx)) = v;
  }
};

// The persistent step over one group of tiles: every instance in a group
// shares the boundary rule (and, for 2-byte formats, the x-pair mapping), so
// the per-cell code is inlined once, exactly as in the single-lattice
// kernels.  Block b takes tiles t0 + b, t0 + b + grid, ... of [t0, t1).
template <Store S, bool EXACT, Bc B, CaseRule RULE, bool X2>
__global__ void __launch_bounds__(256, 2) engine_step_kernel(const EngArgs ea, const int t0, const int t1) {
  using T = typename StoreT<S>::T;
  constexpr int CPT = CellsPerThread<S>::value;
  // raw storage: EngInst has default member initialisers, which a
  // __shared__ variable cannot run; every field is copied in below
  __shared__ __align__(16) unsigned char sh_raw[sizeof(EngInst)];
  EngInst& sh = *reinterpret_cast<EngInst*>(sh_raw);
  int loaded = -1;  // same tile sequence in every thread: a block-uniform value
  for (int t = t0 + blockIdx.x; t < t1; t += gridDim.x) {
    const Tile tile = ea.tiles[t];
    const int left = ea.left[tile.slot];  // block-uniform
    if (left == 0) continue;              // the instance has taken its steps
    if (tile.slot != loaded) {
      __syncthreads();
      const int4* from = reinterpret_cast<const int4*>(ea.inst + tile.slot);
      int4* to = reinterpret_cast<int4*>(&sh);
      for (int w = threadIdx.x; w < static_cast<int>(sizeof(EngInst) / 16); w += blockDim.x) to[w] = from[w];
      __syncthreads();
      if (threadIdx.x == 0) {
        sh.a.store = ea.store || left == 1;
        sh.a.seed = sr_hash(ea.seed[tile.slot]);
      }
      __syncthreads();
      loaded = tile.slot;
    }
    const int cur = (ea.parity ^ sh.parity0) & 1;
    const FlatPlanes<T> pl{static_cast<const T*>(sh.buf[cur]), static_cast<T*>(sh.buf[1 - cur]),
                           static_cast<int32_t>(sh.a.sq)};
    const int bxl = sh.bx_log2;
    const int tx = threadIdx.x & ((1 << bxl) - 1), ty = threadIdx.x >> bxl;
    if constexpr (X2) {
      // 2-byte cavity and sphere instances round stochastically (stochastic_rounding_for)
      step_cells_x2<S, B, RULE, S != Store::F32 && (RULE == CaseRule::CavityStd || RULE == CaseRule::SphereStd)>(
          sh.a, pl, tile.i0 + 2 * tx, tile.j0 + PairRows<S>::value * ty, tile.k);
    } else {
      double drag[3] = {0.0, 0.0, 0.0};
      step_cells<S, B, RULE, EXACT, false>(sh.a, pl, tile.i0 + tx, tile.j0 + ty * CPT, tile.k, drag);
    }
  }
}

// The persistent step over one group of staged tiles (2-byte formats with
// rows staged in shared memory, stage_core.cuh): the single-lattice staged
// kernel's pipeline, where each tile may belong to another instance.  With a
// tile's rows, warp 0 copies the prefix of its instance's StepArgs into the
// stage, so the per-cell code reads the instance's constants from shared
// memory.
template <Store S, Bc B, CaseRule RULE>
__global__ void __launch_bounds__(stage::THREADS, 2) engine_staged_kernel(const EngArgs ea, const int t0,
                                                                          const int t1) {
  using T = typename StoreT<S>::T;
  using namespace stage;
  constexpr bool WRAP = B == Bc::Periodic || RULE == CaseRule::SphereStd;
  constexpr bool REC = RULE == CaseRule::CavityStd;  // wall records staged with the rows
  constexpr int NS = MAX_STAGES;
  constexpr int stage_elems = Q * SLOT_CAP;
  extern __shared__ __align__(128) unsigned char smem[];
  T* stages = reinterpret_cast<T*>(smem);
  unsigned char* args = smem + static_cast<size_t>(Q) * SLOT_UNITS * sizeof(T);
  unsigned char* recs = args + NS * STAGED_ARGS_BYTES;
  TileHdr* hdr = reinterpret_cast<TileHdr*>(recs + (REC ? NS * REC_STAGE_BYTES : 0));
  StagedTile* dslot = reinterpret_cast<StagedTile*>(reinterpret_cast<unsigned char*>(hdr) + NS * TILE_HDR_BYTES);
  uint64_t* full = reinterpret_cast<uint64_t*>(dslot + 2);
  uint64_t* empty = full + NS;
  auto rec_stage = [&](int sn) { return reinterpret_cast<uint16_t*>(recs + sn * REC_STAGE_BYTES); };
  __shared__ int abort_flag;
  if (threadIdx.x == 0) {
    for (int s = 0; s < NS; ++s) {
      bar_init(&full[s], 1);
      bar_init(&empty[s], THREADS / 32);
    }
    abort_flag = 0;
    bar_init_fence();
  }
  __syncthreads();
  volatile int* abort_v = &abort_flag;
  const int grid = gridDim.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  // Warp 0 issues the block's tiles in order t0 + blockIdx.x + n grid.  The
  // descriptor of the next one is copied into shared memory one tile ahead
  // (cp.async, lanes 0-7; tile n of the block uses descriptor slot n & 1),
  // so the copies of a tile wait on no global load.
  auto fetch = [&](int t, int n) {
    if (t < t1 && lane < 8)
      cp_async16(reinterpret_cast<unsigned char*>(dslot + (n & 1)) + 16 * lane,
                 reinterpret_cast<const unsigned char*>(ea.stiles + t) + 16 * lane);
  };
  int issued = 0;
  // copies of the block's tile number `issued` into stage sn (warp 0), then
  // fetch the descriptor of the next one, tile tf
  auto issue = [&](int sn, int tf) {
    cp_async_wait_all();
    __syncwarp();
    const StagedTile& d = dslot[issued & 1];
    const int cur = (ea.parity ^ d.parity0) & 1;
    const void* src_buf = d.buf[cur];
    const int left = ea.left[d.slot];
    if (lane == 0)
      hdr[sn] = TileHdr{src_buf, const_cast<void*>(d.buf[1 - cur]), REC ? d.rec[1 - cur] : nullptr, d.geo, d.j0,
                        d.k, left == 0, ea.store || left == 1, sr_hash(ea.seed[d.slot])};
    if (left == 0)
      issue_skip(&full[sn]);
    else
      issue_tile<T, WRAP>(d, d.geo, static_cast<const T*>(src_buf), d.j0, d.k, stages + sn * stage_elems, &full[sn],
                          REC ? d.rec[cur] : nullptr, rec_stage(sn), args + sn * STAGED_ARGS_BYTES, d.args,
                          static_cast<uint32_t>(STAGED_ARGS_BYTES));
    __syncwarp();  // every lane has read the slot before the fetch after next refills it
    fetch(tf, issued + 1);
  };
  if (warp == 0) fetch(t0 + blockIdx.x, 0);
  if (warp == 0) {
    for (; issued < NS - 1; ++issued) {
      const int t = t0 + blockIdx.x + issued * grid;
      if (t >= t1) break;
      issue(issued, t + grid);
    }
  }
  int i = 0;
  for (int t = t0 + blockIdx.x; t < t1; t += grid, ++i) {
    const int s = i % NS;
    if (warp == 0) {
      const int tn = t + (NS - 1) * grid;
      if (tn < t1) {
        if (i > 0 && !__all_sync(0xffffffffu, bar_wait(&empty[(i - 1) % NS], ((i - 1) / NS) & 1u))) {
          *abort_v = 1;
          break;
        }
        issue((i + NS - 1) % NS, tn + grid);
        ++issued;
      }
    }
    if (!__all_sync(0xffffffffu, bar_wait(&full[s], (i / NS) & 1u))) {
      *abort_v = 1;
      break;
    }
    const TileHdr& h = hdr[s];
    if (!h.skip) {
      const StepArgs& a = *reinterpret_cast<const StepArgs*>(args + s * STAGED_ARGS_BYTES);
      // the cavity and the vortex: one 64-bit plane base a pair and the
      // block-uniform offset q * sq a population; the sphere's kernels keep
      // 32-bit plane indices (they spill 56 bytes with the 64-bit base)
      using PL = std::conditional_t<RULE == CaseRule::SphereStd, FlatPlanes<T>, StridedPlanes<T>>;
      const PL pl{static_cast<const T*>(h.src), static_cast<T*>(h.dst),
                  static_cast<decltype(PL::sq)>(a.sq)};
      const Geo g = h.geo;
      consume_tile<S, B, RULE, RULE == CaseRule::CavityStd || RULE == CaseRule::SphereStd>(
          a, pl, g, reinterpret_cast<const uint32_t*>(stages + s * stage_elems), h.j0, h.k, h.store != 0, h.seed,
          rec_stage(s), h.rec);
    }
    __syncwarp();
    if (lane == 0) bar_arrive(&empty[s]);
    if (__any_sync(0xffffffffu, *abort_v != 0)) break;
  }
  if (warp == 0 && lane == 0 && *abort_v) {
    for (int m = i; m < issued; ++m) (void)bar_wait(&full[m % NS], (m / NS) & 1u);
  }
  __syncthreads();
  if (threadIdx.x == 0 && abort_flag) atomicOr(ea.err, 1);
}

inline size_t engine_staged_smem(bool records) {
  return static_cast<size_t>(Q) * stage::SLOT_UNITS * 2 + stage::MAX_STAGES * STAGED_ARGS_BYTES +
         (records ? stage::MAX_STAGES * stage::REC_STAGE_BYTES : 0) + stage::MAX_STAGES * TILE_HDR_BYTES +
         2 * sizeof(StagedTile) + 16 * stage::MAX_STAGES;
}

// Residual partial sums per tile: sum |u - u_prev|^2 and sum |u|^2 over the
// tile's cells, then u_prev = u.  Deterministic: per-tile partials are added
// in tile order per instance afterwards.
__global__ void engine_resid_kernel(const EngArgs ea, double* part) {
  __shared__ double sh[2][8];
  for (int t = blockIdx.x; t < ea.ntiles; t += gridDim.x) {
    const Tile tile = ea.tiles[t];
    const EngInst& in = ea.inst[tile.slot];
    const int k = tile.k;
    const int nx = in.a.nx, ny = in.a.ny;
    const bool flat = in.staged && in.geo.flat;  // flat tiles: j0 is the tile's first element
    const int tw = flat ? in.geo.C : in.tw, th = flat ? 1 : in.th;
    const int64_t n = static_cast<int64_t>(nx) * ny * in.a.nz;
    double d2 = 0.0, n2 = 0.0;
    for (int c = threadIdx.x; c < tw * th; c += blockDim.x) {
      int i = tile.i0 + c % tw, j = tile.j0 + c / tw;
      if (flat) {
        const int e = tile.j0 + c;
        j = e / in.geo.P;
        i = e - j * in.geo.P;
      }
      if (i < nx && j < ny) {
        const int64_t cell = i + static_cast<int64_t>(nx) * (j + static_cast<int64_t>(ny) * k);
        const double u = in.a.mu[cell], v = in.a.mv[cell], w = in.a.mw[cell];
        double* pu = in.prev + cell;
        double* pv = in.prev + n + cell;
        double* pw = in.prev + 2 * n + cell;
        const double du = u - *pu, dv = v - *pv, dw = w - *pw;
        d2 += du * du + dv * dv + dw * dw;
        n2 += u * u + v * v + w * w;
        *pu = u;
        *pv = v;
        *pw = w;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      d2 += __shfl_xor_sync(0xffffffffu, d2, o);
      n2 += __shfl_xor_sync(0xffffffffu, n2, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) {
      sh[0][warp] = d2;
      sh[1][warp] = n2;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
      double x = 0.0;
      for (int w = 0; w < 8; ++w) x += sh[threadIdx.x][w];
      part[2 * static_cast<int64_t>(t) + threadIdx.x] = x;
    }
  }
}

// One block per listed instance: add its tiles' partials in order.
__global__ void engine_resid_reduce(const int* seg_begin, const int* seg_end, const double* part, double* out) {
  const int s = blockIdx.x;
  double d2 = 0.0, n2 = 0.0;
  for (int t = seg_begin[s] + threadIdx.x; t < seg_end[s]; t += blockDim.x) {
    d2 += part[2 * static_cast<int64_t>(t)];
    n2 += part[2 * static_cast<int64_t>(t) + 1];
  }
  __shared__ double sh[2][8];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    d2 += __shfl_xor_sync(0xffffffffu, d2, o);
    n2 += __shfl_xor_sync(0xffffffffu, n2, o);
  }
  if ((threadIdx.x & 31) == 0) {
    sh[0][threadIdx.x >> 5] = d2;
    sh[1][threadIdx.x >> 5] = n2;
  }
  __syncthreads();
  if (threadIdx.x < 2) {
    double x = 0.0;
    for (int w = 0; w < 8; ++w) x += sh[threadIdx.x][w];
    out[2 * s + threadIdx.x] = x;
  }
}

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t cap = 0;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  cudaError_t reserve(size_t n) {
    if (n <= cap) return cudaSuccess;
    const size_t want = std::max(n, cap + cap / 2);
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&p), want * sizeof(T));
    if (e == cudaSuccess) cap = want;
    return e;
  }
};

// First-fit arena over one device allocation, 512-byte granules, with
// coalescing of freed neighbours.
class Arena {
 public:
  char* base = nullptr;
  size_t size = 0;
  std::map<size_t, size_t> free_;  // offset -> length
  size_t used = 0;
  bool alloc(size_t bytes, size_t* off) {
    bytes = (bytes + 511) & ~static_cast<size_t>(511);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < bytes) continue;
      *off = it->first;
      const size_t rest = it->second - bytes;
      const size_t o = it->first;
      free_.erase(it);
      if (rest) free_[o + bytes] = rest;
      used += bytes;
      return true;
    }
    return false;
  }
  void release(size_t off, size_t bytes) {
    bytes = (bytes + 511) & ~static_cast<size_t>(511);
    used -= bytes;
    auto it = free_.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
};

struct Slot {
  bool used = false;
  imexlb_storage storage = IMEXLB_F64;  // the instance's own storage format
  imexlb_instance_desc d{};
  Layout L;
  size_t off = 0, bytes = 0;
  int64_t ncell = 0;
  int64_t steps = 0;
  int64_t run = 0;  // steps taken since admission (its buffer parity)
  int64_t run_checked = -1;  // `run` at the last residual check
  bool have_prev = false;
  int bx_log2 = 5;
  int seg = -1;  // index into the segment table of the current work list
};

int bx_log2_for(int nx, int tile_bx) {
  int bx = tile_bx;
  if (bx <= 0) {
    bx = 16;
    while (bx < nx && bx < 128) bx *= 2;
  }
  int l = 0;
  while ((1 << l) < bx) ++l;
  return std::min(std::max(l, 3), 8);
}

// Pinned host buffers for the uploads of engine_add: an admission copies its
// initial fields through one of them and returns without waiting; a buffer
// is reused once the event recorded after its copies has completed.
class Staging {
 public:
  ~Staging() {
    for (auto& b : bufs_) {
      if (b.ev) cudaEventDestroy(b.ev);
      if (b.p) cudaFreeHost(b.p);
    }
  }
  // a free buffer of at least n bytes (index into the pool), or -1
  int get(size_t n, cudaError_t* err) {
    int best = -1;
    for (int i = 0; i < static_cast<int>(bufs_.size()); ++i) {
      Buf& b = bufs_[i];
      if (b.busy && cudaEventQuery(b.ev) == cudaSuccess) b.busy = false;
      if (!b.busy && b.cap >= n && (best < 0 || b.cap < bufs_[best].cap)) best = i;
    }
    *err = cudaSuccess;
    if (best >= 0) return best;
    Buf b;
    const size_t cap = std::max(n, static_cast<size_t>(1) << 20);
    if ((*err = cudaMallocHost(reinterpret_cast<void**>(&b.p), cap)) != cudaSuccess) return -1;
    if ((*err = cudaEventCreateWithFlags(&b.ev, cudaEventDisableTiming)) != cudaSuccess) {
      cudaFreeHost(b.p);
      return -1;
    }
    b.cap = cap;
    bufs_.push_back(b);
    return static_cast<int>(bufs_.size()) - 1;
  }
  char* ptr(int i) { return bufs_[i].p; }
  cudaError_t release_after(int i, cudaStream_t s) {
    bufs_[i].busy = true;
    return cudaEventRecord(bufs_[i].ev, s);
  }

 private:
  struct Buf {
    char* p = nullptr;
    size_t cap = 0;
    cudaEvent_t ev = nullptr;
    bool busy = false;
  };
  std::vector<Buf> bufs_;
};

}  // namespace
}  // namespace imx

using namespace imx;

struct imexlb_engine {
  Staging staging;  // pinned uploads of admissions (declared first: destroyed last)
  imexlb_storage storage = IMEXLB_F64;
  bool exact = false;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  Arena arena;
  std::vector<Slot> slots;
  std::vector<EngInst> h_inst;
  DevBuf<EngInst> d_inst;
  DevBuf<Tile> d_tiles;
  std::vector<Tile> h_tiles;
  DevBuf<StagedTile> d_stiles;
  std::vector<StagedTile> h_stiles;
  DevBuf<int> d_left;       // per slot: steps left (ENG_NO_LIMIT: no limit)
  DevBuf<uint32_t> d_taken; // per slot: steps taken (counted on the device by engine_tick)
  std::vector<int> h_left;  // host copy, counted down with the steps run
  DevBuf<double> d_part;
  DevBuf<int> d_seg;  // begin[nseg], end[nseg]
  DevBuf<double> d_res;
  std::vector<int> seg_slots;
  // tile ranges of the kernel groups: group = storage format * 9 + rule (0
  // periodic, 1 cavity, 2 sphere) * 3 + mode (0 one cell or y-pairs, 1
  // x-pairs, 2 staged rows)
  static constexpr int GROUPS = 4 * 9;
  int group_begin[GROUPS] = {};
  int group_end[GROUPS] = {};
  DevBuf<int> d_err;  // staged kernels' error word
  int staged_resident = 0;  // staged blocks resident on the device
  bool staged_ready[4] = {};  // staged kernels' shared memory set for this format
  bool dirty = true;
  int64_t gstep = 0;
  int grid = 296;
  cudaGraphExec_t graph = nullptr;
  int graph_tiles = -1;
  bool use_graph = true;
  ~imexlb_engine() {
    if (graph) cudaGraphExecDestroy(graph);
    if (arena.base) cudaFree(arena.base);
    if (own_stream && stream) cudaStreamDestroy(stream);
  }
};

namespace {

int efail(int code, const std::string& msg) { return imx::set_last_error(code, msg); }

#define IMX_ECUDA(call)                                                                        \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess) return efail(IMEXLB_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

int cpt_of(imexlb_storage s) { return s == IMEXLB_F64 ? 1 : 2; }

// Wait for the engine's stream and report a staged kernel that gave up
// waiting for its row copies (the error word is then cleared).
int sync_checked(imexlb_engine* e) {
  int word = 0;
  IMX_ECUDA(cudaMemcpyAsync(&word, e->d_err.p, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
  IMX_ECUDA(cudaStreamSynchronize(e->stream));
  if (word) {
    IMX_ECUDA(cudaMemset(e->d_err.p, 0, sizeof(int)));
    return efail(IMEXLB_E_CUDA, "a staged step kernel gave up waiting for its row copies; instance states are invalid");
  }
  return IMEXLB_OK;
}

int mode_of(const EngInst& in) { return in.staged ? 2 : (in.x2 ? 1 : 0); }
int group_of(const Slot& sl, const EngInst& in) {
  const int rule = in.rule;
  const int rg = rule == static_cast<int>(CaseRule::None) ? 0 : (rule == static_cast<int>(CaseRule::CavityStd) ? 1 : 2);
  return static_cast<int>(sl.storage) * 9 + rg * 3 + mode_of(in);
}

int rebuild_tiles(imexlb_engine* e) {
  if (!e->dirty) return IMEXLB_OK;
  e->h_tiles.clear();
  e->seg_slots.clear();
  std::vector<int> sb, se;
  // instances ordered by kernel group, so that each group's tiles are one range
  std::vector<int> order;
  for (int g = 0; g < imexlb_engine::GROUPS; ++g)
    for (int s = 0; s < static_cast<int>(e->slots.size()); ++s)
      if (e->slots[s].used && group_of(e->slots[s], e->h_inst[s]) == g) order.push_back(s);
  for (int g = 0; g < imexlb_engine::GROUPS; ++g) e->group_begin[g] = e->group_end[g] = 0;
  int prev_group = -1;
  for (int s : order) {
    Slot& sl = e->slots[s];
    const EngInst& in = e->h_inst[s];
    const int g = group_of(sl, in);
    if (g != prev_group) {
      e->group_begin[g] = static_cast<int>(e->h_tiles.size());
      prev_group = g;
    }
    sl.seg = static_cast<int>(e->seg_slots.size());
    e->seg_slots.push_back(s);
    sb.push_back(static_cast<int>(e->h_tiles.size()));
    if (in.staged && in.geo.flat) {
      // flat tiles (stage_core.cuh): j0 holds the tile's first element of its plane
      for (int k = 0; k < sl.L.nz; ++k)
        for (int t = 0; t < in.geo.nty; ++t) e->h_tiles.push_back(Tile{s, 0, t * in.geo.C, k});
    } else {
      for (int k = 0; k < sl.L.nz; ++k)
        for (int j0 = 0; j0 < sl.L.ny; j0 += in.th)
          for (int i0 = 0; i0 < sl.L.nx; i0 += in.tw) e->h_tiles.push_back(Tile{s, i0, j0, k});
    }
    se.push_back(static_cast<int>(e->h_tiles.size()));
    e->group_end[g] = static_cast<int>(e->h_tiles.size());
  }
  const size_t nt = e->h_tiles.size();
  // staged tiles: the flattened descriptors their kernels' warp 0 reads
  e->h_stiles.assign(nt, StagedTile{});
  for (size_t t = 0; t < nt; ++t) {
    const Tile& tl = e->h_tiles[t];
    const EngInst& in = e->h_inst[tl.slot];
    if (!in.staged) continue;
    StagedTile& d = e->h_stiles[t];
    d.buf[0] = in.buf[0];
    d.buf[1] = in.buf[1];
    d.rec[0] = in.rec[0];
    d.rec[1] = in.rec[1];
    d.args = &(e->d_inst.p + tl.slot)->a;
    d.sq = in.a.sq;
    d.base32 = in.a.base32;
    d.sz32 = in.a.sz32;
    d.pitch32 = in.a.pitch32;
    d.nx = in.a.nx;
    d.ny = in.a.ny;
    d.nz = in.a.nz;
    d.parity0 = in.parity0;
    d.j0 = tl.j0;
    d.k = tl.k;
    d.geo = in.geo;
    d.slot = tl.slot;
  }
  if (nt) {
    IMX_ECUDA(e->d_tiles.reserve(nt));
    IMX_ECUDA(cudaMemcpyAsync(e->d_tiles.p, e->h_tiles.data(), nt * sizeof(Tile), cudaMemcpyHostToDevice, e->stream));
    IMX_ECUDA(e->d_stiles.reserve(nt));
    IMX_ECUDA(cudaMemcpyAsync(e->d_stiles.p, e->h_stiles.data(), nt * sizeof(StagedTile), cudaMemcpyHostToDevice,
                              e->stream));
    IMX_ECUDA(e->d_part.reserve(2 * nt));
  }
  const size_t ns = e->seg_slots.size();
  if (ns) {
    std::vector<int> seg(2 * ns);
    std::copy(sb.begin(), sb.end(), seg.begin());
    std::copy(se.begin(), se.end(), seg.begin() + ns);
    IMX_ECUDA(e->d_seg.reserve(2 * ns));
    IMX_ECUDA(cudaMemcpyAsync(e->d_seg.p, seg.data(), seg.size() * sizeof(int), cudaMemcpyHostToDevice, e->stream));
    IMX_ECUDA(e->d_res.reserve(2 * ns));
  }
  IMX_ECUDA(cudaStreamSynchronize(e->stream));  // host vectors may change before the next call
  e->dirty = false;
  if (e->graph) {
    cudaGraphExecDestroy(e->graph);
    e->graph = nullptr;
  }
  return IMEXLB_OK;
}

template <Store S>
void set_staged_smem() {
  const int smem = static_cast<int>(engine_staged_smem(false));
  cudaFuncSetAttribute(engine_staged_kernel<S, Bc::Periodic, CaseRule::None>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  cudaFuncSetAttribute(engine_staged_kernel<S, Bc::Standard, CaseRule::CavityStd>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(engine_staged_smem(true)));
  cudaFuncSetAttribute(engine_staged_kernel<S, Bc::Standard, CaseRule::SphereStd>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
}

// The kernel groups of the instances stored in format S.
template <Store S, bool EXACT>
cudaError_t launch_groups(const imexlb_engine* e, const EngArgs& ea) {
  for (int g = 0; g < 9; ++g) {
    const int t0 = e->group_begin[static_cast<int>(S) * 9 + g], t1 = e->group_end[static_cast<int>(S) * 9 + g];
    if (t1 <= t0) continue;
    const int rule = g / 3, mode = g % 3;
    if constexpr (S == Store::F16 || S == Store::BF16) {
      if (mode == 2) {
        const int grid = std::min(e->staged_resident, t1 - t0);
        const size_t smem = engine_staged_smem(rule == 1);
        if (rule == 0)
          engine_staged_kernel<S, Bc::Periodic, CaseRule::None><<<grid, stage::THREADS, smem, e->stream>>>(ea, t0, t1);
        else if (rule == 1)
          engine_staged_kernel<S, Bc::Standard, CaseRule::CavityStd><<<grid, stage::THREADS, smem, e->stream>>>(ea, t0,
                                                                                                                 t1);
        else
          engine_staged_kernel<S, Bc::Standard, CaseRule::SphereStd><<<grid, stage::THREADS, smem, e->stream>>>(ea, t0,
                                                                                                                 t1);
        continue;
      }
      if (mode == 1) {
        const int grid = std::min(e->grid, t1 - t0);
        if (rule == 0)
          engine_step_kernel<S, false, Bc::Periodic, CaseRule::None, true><<<grid, 256, 0, e->stream>>>(ea, t0, t1);
        else if (rule == 1)
          engine_step_kernel<S, false, Bc::Standard, CaseRule::CavityStd, true><<<grid, 256, 0, e->stream>>>(ea, t0, t1);
        else
          engine_step_kernel<S, false, Bc::Standard, CaseRule::SphereStd, true><<<grid, 256, 0, e->stream>>>(ea, t0, t1);
        continue;
      }
    }
    if constexpr (S == Store::F32) {
      // FP32 x-pairs (the vortex)
      if (mode == 1 && rule == 0) {
        const int grid = std::min(e->grid, t1 - t0);
        engine_step_kernel<S, false, Bc::Periodic, CaseRule::None, true><<<grid, 256, 0, e->stream>>>(ea, t0, t1);
        continue;
      }
    }
    const int grid = std::min(e->grid, t1 - t0);
    if (rule == 0)
      engine_step_kernel<S, EXACT, Bc::Periodic, CaseRule::None, false><<<grid, 256, 0, e->stream>>>(ea, t0, t1);
    else if (rule == 1)
      engine_step_kernel<S, EXACT, Bc::Standard, CaseRule::CavityStd, false><<<grid, 256, 0, e->stream>>>(ea, t0, t1);
    else
      engine_step_kernel<S, EXACT, Bc::Standard, CaseRule::SphereStd, false><<<grid, 256, 0, e->stream>>>(ea, t0, t1);
  }
  return cudaGetLastError();
}

cudaError_t launch_engine(const imexlb_engine* e, int parity, int store) {
  EngArgs ea{e->d_inst.p, e->d_tiles.p, e->d_stiles.p, e->d_left.p, static_cast<int>(e->h_tiles.size()), parity,
              store, e->d_err.p, e->d_taken.p};
  if (ea.ntiles == 0) return cudaSuccess;
  // one pass per storage format present (instances of several formats share
  // the engine and its step graph)
  auto present = [&](int st) {
    for (int g = 0; g < 9; ++g)
      if (e->group_end[st * 9 + g] > e->group_begin[st * 9 + g]) return true;
    return false;
  };
  cudaError_t err = cudaSuccess;
  if (present(IMEXLB_F64))
    err = e->exact ? launch_groups<Store::F64, true>(e, ea) : launch_groups<Store::F64, false>(e, ea);
  if (err == cudaSuccess && present(IMEXLB_F32)) err = launch_groups<Store::F32, false>(e, ea);
  if (err == cudaSuccess && present(IMEXLB_F16)) err = launch_groups<Store::F16, false>(e, ea);
  if (err == cudaSuccess && present(IMEXLB_BF16)) err = launch_groups<Store::BF16, false>(e, ea);
  if (err != cudaSuccess) return err;
  const int n = static_cast<int>(e->h_left.size());
  engine_tick<<<(n + 255) / 256, 256, 0, e->stream>>>(e->d_left.p, e->d_taken.p, n);
  return cudaGetLastError();
}

}  // namespace

// The staged kernels of a 2-byte format: their shared memory is set, and
// their resident blocks counted, once per engine and format (outside any
// stream capture: at creation or at the first admission in the format).
static int prepare_storage(imexlb_engine* e, imexlb_storage storage) {
  if ((storage != IMEXLB_F16 && storage != IMEXLB_BF16) || e->staged_ready[storage]) return IMEXLB_OK;
  int dev = 0, sms = 148, per_sm = 0;
  IMX_ECUDA(cudaGetDevice(&dev));
  IMX_ECUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  if (storage == IMEXLB_F16) {
    set_staged_smem<Store::F16>();
    IMX_ECUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, engine_staged_kernel<Store::F16, Bc::Standard, CaseRule::CavityStd>, stage::THREADS,
        engine_staged_smem(true)));
  } else {
    set_staged_smem<Store::BF16>();
    IMX_ECUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, engine_staged_kernel<Store::BF16, Bc::Standard, CaseRule::CavityStd>, stage::THREADS,
        engine_staged_smem(true)));
  }
  const int resident = std::max(per_sm, 1) * sms;
  e->staged_resident = e->staged_resident ? std::min(e->staged_resident, resident) : resident;
  e->staged_ready[storage] = true;
  return IMEXLB_OK;
}

extern "C" {

int imexlb_engine_create(imexlb_storage storage, imexlb_arith arith, size_t budget_bytes, int max_instances,
                         void* stream, imexlb_engine** out) {
  if (!out) return efail(IMEXLB_E_ARG, "null output");
  *out = nullptr;
  if (storage < IMEXLB_F64 || storage > IMEXLB_BF16) return efail(IMEXLB_E_ARG, "unknown storage");
  if (max_instances < 1 || max_instances > 65536) return efail(IMEXLB_E_ARG, "max_instances must be 1..65536");
  if (budget_bytes < (size_t(1) << 20)) return efail(IMEXLB_E_ARG, "budget below 1 MiB");
  std::unique_ptr<imexlb_engine> e(new imexlb_engine);
  e->storage = storage;
  e->exact = storage == IMEXLB_F64 && arith == IMEXLB_ARITH_EXACT;
  if (stream) {
    e->stream = static_cast<cudaStream_t>(stream);
  } else {
    IMX_ECUDA(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
    e->own_stream = true;
  }
  void* base = nullptr;
  IMX_ECUDA(cudaMalloc(&base, budget_bytes));
  e->arena.base = static_cast<char*>(base);
  e->arena.size = budget_bytes;
  e->arena.free_[0] = budget_bytes & ~static_cast<size_t>(511);
  e->slots.resize(max_instances);
  e->h_inst.resize(max_instances);
  IMX_ECUDA(e->d_inst.reserve(max_instances));
  e->h_left.assign(max_instances, ENG_NO_LIMIT);
  IMX_ECUDA(e->d_left.reserve(max_instances));
  IMX_ECUDA(e->d_taken.reserve(max_instances));
  IMX_ECUDA(cudaMemset(e->d_taken.p, 0, max_instances * sizeof(uint32_t)));
  IMX_ECUDA(cudaMemcpy(e->d_left.p, e->h_left.data(), max_instances * sizeof(int), cudaMemcpyHostToDevice));
  int dev = 0, sms = 148;
  IMX_ECUDA(cudaGetDevice(&dev));
  IMX_ECUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  e->grid = 2 * sms;
  IMX_ECUDA(e->d_err.reserve(1));
  IMX_ECUDA(cudaMemset(e->d_err.p, 0, sizeof(int)));
  if (const int rc = prepare_storage(e.get(), storage)) return rc;
  *out = e.release();
  return IMEXLB_OK;
}

static CaseRule rule_of_case(int kase) {
  return kase == IMEXLB_TGV ? CaseRule::None : (kase == IMEXLB_CAVITY ? CaseRule::CavityStd : CaseRule::SphereStd);
}

// Rows of the instance staged in shared memory (2-byte formats, nx even,
// rows that fit a stage and no register-staged tile width asked for).
static bool instance_staged(int storage, const imexlb_instance_desc* d, const Layout& L, stage::Geo* g) {
  const bool x2 = (storage == IMEXLB_F16 || storage == IMEXLB_BF16) && d->nx % 2 == 0;
  return x2 && d->tile_bx <= 0 && stage::staged_layout(rule_of_case(d->kase), d->nx, d->ny, L.pitch, g);
}

// Bytes of one wall-record buffer of the instance (a staged cavity), else 0.
static size_t record_bytes(int storage, const imexlb_instance_desc* d, const Layout& L) {
  stage::Geo g;
  if (d->kase != IMEXLB_CAVITY || !instance_staged(storage, d, L, &g)) return 0;
  return (static_cast<size_t>(d->ny) * d->nz * WallRecord::BYTES + 511) & ~static_cast<size_t>(511);
}

int imexlb_engine_add(imexlb_engine* e, const imexlb_instance_desc* d, int* slot_out) {
  if (!e) return efail(IMEXLB_E_ARG, "null engine");
  return imexlb_engine_add_as(e, d, e->storage, slot_out);
}

int imexlb_engine_add_as(imexlb_engine* e, const imexlb_instance_desc* d, imexlb_storage storage, int* slot_out) {
  if (!e || !d || !slot_out) return efail(IMEXLB_E_ARG, "null argument");
  if (storage < IMEXLB_F64 || storage > IMEXLB_BF16) return efail(IMEXLB_E_ARG, "unknown storage");
  if (const int rc = prepare_storage(e, storage)) return rc;
  if (d->kase != IMEXLB_TGV && d->kase != IMEXLB_CAVITY && d->kase != IMEXLB_SPHERE)
    return efail(IMEXLB_E_ARG, "unknown case");
  if (d->nx < 2 || d->ny < 2 || d->nz < 2 || d->nz > 65535) return efail(IMEXLB_E_ARG, "bad extents");
  if (!(d->tau0 > 0.0)) return efail(IMEXLB_E_ARG, "tau0 must be positive");
  int s = -1;
  for (int i = 0; i < static_cast<int>(e->slots.size()); ++i)
    if (!e->slots[i].used) {
      s = i;
      break;
    }
  if (s < 0) return efail(IMEXLB_E_NOMEM, "no free instance slot");
  const int elem = storage == IMEXLB_F64 ? 8 : (storage == IMEXLB_F32 ? 4 : 2);
  Slot sl;
  sl.storage = storage;
  sl.d = *d;
  sl.L = make_layout(d->nx, d->ny, d->nz, 0, elem);
  if (static_cast<double>(sl.L.sq) * Q >= 2147483647.0) return efail(IMEXLB_E_ARG, "instance too large for the engine");
  sl.ncell = static_cast<int64_t>(d->nx) * d->ny * d->nz;
  const size_t fbytes = (sl.L.bytes() + 511) & ~static_cast<size_t>(511);
  const size_t mbytes = ((4 * sl.ncell * 8) + 511) & ~static_cast<size_t>(511);
  const size_t pbytes = ((3 * sl.ncell * 8) + 511) & ~static_cast<size_t>(511);
  const size_t mask_bytes = static_cast<size_t>((sl.ncell + 255) & ~int64_t(255));
  const size_t sbytes = d->kase == IMEXLB_SPHERE ? ((mask_bytes + 4 * sl.ncell + 511) & ~static_cast<size_t>(511)) : 0;
  const size_t rbytes = record_bytes(storage, d, sl.L);
  sl.bytes = 2 * fbytes + mbytes + pbytes + sbytes + 2 * rbytes;
  if (!e->arena.alloc(sl.bytes, &sl.off))
    return efail(IMEXLB_E_NOMEM, "instance does not fit the engine's memory budget");
  char* b = e->arena.base + sl.off;
  void* buf0 = b;
  void* buf1 = b + fbytes;
  double* mom = reinterpret_cast<double*>(b + 2 * fbytes);
  double* prev = reinterpret_cast<double*>(b + 2 * fbytes + mbytes);
  uint8_t* usr = d->kase == IMEXLB_SPHERE ? reinterpret_cast<uint8_t*>(b + 2 * fbytes + mbytes + pbytes) : nullptr;
  uint32_t* links = usr ? reinterpret_cast<uint32_t*>(usr + mask_bytes) : nullptr;
  uint16_t* rec0 = rbytes ? reinterpret_cast<uint16_t*>(b + 2 * fbytes + mbytes + pbytes + sbytes) : nullptr;
  uint16_t* rec1 = rbytes ? reinterpret_cast<uint16_t*>(b + 2 * fbytes + mbytes + pbytes + sbytes + rbytes) : nullptr;

  // initial fields (the same set-up as a single lattice)
  imexlb_params P;
  imexlb_params_default(&P);
  P.kase = d->kase;
  P.bc = d->kase == IMEXLB_TGV ? IMEXLB_BC_REFERENCE : IMEXLB_BC_STANDARD;
  P.storage = storage;
  P.nx = d->nx;
  P.ny = d->ny;
  P.nz = d->nz;
  P.tau0 = d->tau0;
  P.rho0 = d->rho0;
  P.u0 = d->u0;
  P.lid_u = d->lid_u != 0.0 ? d->lid_u : d->u0;
  P.inlet_u = d->inlet_u != 0.0 ? d->inlet_u : d->u0;
  P.sphere_d = d->sphere_d != 0.0 ? d->sphere_d : d->nx / 24.0;
  P.sphere_c[0] = d->sphere_c[0];
  P.sphere_c[1] = d->sphere_c[1];
  P.sphere_c[2] = d->sphere_c[2];
  if (d->kase == IMEXLB_SPHERE && P.sphere_c[0] == 0.0 && P.sphere_c[1] == 0.0 && P.sphere_c[2] == 0.0) {
    P.sphere_c[0] = d->nx / 4.0;
    P.sphere_c[1] = d->ny / 2.0;
    P.sphere_c[2] = d->nz / 2.0;
  }
  const size_t n = static_cast<size_t>(sl.ncell);
  // everything this admission uploads goes through one pinned buffer: the
  // vortex's initial moments (the cavity starts at rest and the sphere
  // channel's fields follow from its mask, both set on the device), then
  // (sphere) mask and links, then the instance descriptor
  const size_t up_mom = d->kase == IMEXLB_TGV ? 4 * n * 8 : 0, up_mask = d->kase == IMEXLB_SPHERE ? n : 0;
  const size_t up_links = d->kase == IMEXLB_SPHERE ? 4 * n : 0;
  const size_t off_links = (up_mom + up_mask + 15) & ~static_cast<size_t>(15);
  const size_t off_inst = (off_links + up_links + 15) & ~static_cast<size_t>(15);
  cudaError_t serr = cudaSuccess;
  const int sb = e->staging.get(off_inst + sizeof(EngInst), &serr);
  if (sb < 0) {
    e->arena.release(sl.off, sl.bytes);
    return efail(IMEXLB_E_NOMEM, std::string("pinned upload buffer: ") + cudaGetErrorString(serr));
  }
  char* up = e->staging.ptr(sb);
  if (d->kase == IMEXLB_TGV) {
    // the initial u, v, w, p straight into the pinned buffer
    std::vector<int32_t> no_mask;
    case_fields(P, sl.L, nullptr, &no_mask, reinterpret_cast<double*>(up));
    IMX_ECUDA(cudaMemcpyAsync(mom, up, up_mom, cudaMemcpyHostToDevice, e->stream));
  } else if (d->kase == IMEXLB_CAVITY) {
    IMX_ECUDA(cudaMemsetAsync(mom, 0, 4 * n * 8, e->stream));  // at rest: u = p = 0
  }

  EngInst& in = e->h_inst[s];
  in = EngInst{};
  StepArgs& a = in.a;
  a.nx = d->nx;
  a.ny = d->ny;
  a.nz = d->nz;
  a.sq = sl.L.sq;
  a.sz = sl.L.sz;
  a.pitch = sl.L.pitch;
  a.base = sl.L.idx(0, 0, 0, 0);
  for (int q = 0; q < Q; ++q) {
    a.rel[q] = static_cast<int32_t>(-(D3Q27::ez[q] * sl.L.sz + D3Q27::ey[q] * sl.L.pitch + D3Q27::ex[q]));
    a.off[q] = q * sl.L.sq + a.rel[q];
  }
  a.base32 = static_cast<int32_t>(a.base);
  a.sz32 = static_cast<int32_t>(sl.L.sz);
  a.pitch32 = static_cast<int32_t>(sl.L.pitch);
  a.tau_half = d->tau0 + 0.5;
  a.omega = 1.0 / (d->tau0 + 0.5);
  a.mu = mom;
  a.mv = mom + n;
  a.mw = mom + 2 * n;
  a.mp = mom + 3 * n;
  a.lid_u = P.lid_u;
  a.rho_w = P.rho0;
  a.inlet_u = P.inlet_u;
  const double p_rest = d->kase == IMEXLB_TGV ? d->rho0 / 3.0 : 0.0;
  a.p_shift = storage == IMEXLB_F64 ? 0.0 : p_rest;
  for (int q = 0; q < Q; ++q) {
    const double sc = store_scale(static_cast<Store>(storage), D3Q27::wclass[q]);
    a.enc.scale[q] = static_cast<float>(sc);
    a.enc.inv_scale[q] = static_cast<float>(1.0 / sc);
  }
  a.enc.unit = store_unit(static_cast<Store>(storage));
  a.enc.sr = stochastic_rounding_for(d->kase, storage);
  in.rule = static_cast<int>(d->kase == IMEXLB_TGV ? CaseRule::None
                                                   : (d->kase == IMEXLB_CAVITY ? CaseRule::CavityStd : CaseRule::SphereStd));
  if (d->kase == IMEXLB_SPHERE) {
    uint8_t* m = reinterpret_cast<uint8_t*>(up + up_mom);
    std_sphere_mask(P, m);
    std::vector<uint32_t> lk;
    int lo[3], hi[3];
    solid_links(d->nx, d->ny, d->nz, m, lk, lo, hi);
    std::memcpy(up + off_links, lk.data(), n * 4);
    IMX_ECUDA(cudaMemcpyAsync(usr, m, n, cudaMemcpyHostToDevice, e->stream));
    IMX_ECUDA(cudaMemcpyAsync(links, up + off_links, n * 4, cudaMemcpyHostToDevice, e->stream));
    IMX_ECUDA(launch_sphere_fields(usr, sl.ncell, P.inlet_u, mom, e->stream));
    a.usr = usr;
    a.links = links;
    for (int c = 0; c < 3; ++c) {
      a.near_lo[c] = lo[c];
      a.near_hi[c] = hi[c];
    }
    const double ui = P.inlet_u;
    // 2-byte x-pair formats store deviations from the inflow's equilibrium
    const bool ref_flow = (storage == IMEXLB_F16 || storage == IMEXLB_BF16) && d->nx % 2 == 0;
    if (ref_flow) set_reference_flow(a.enc, ui, a.omega);
    for (int q = 0; q < Q; ++q) {
      const double t = weight_of_class(D3Q27::wclass[q]);
      const double ev = D3Q27::ex[q] * ui;
      // the reference's equilibrium bracket (tgv/src/lbm.cpp:228-232) of (ui, 0, 0): edu = e_x ui, udu = ui ui
      const double br = 3.0 * ev + 4.5 * (ev * ev) - 1.5 * (ui * ui);
      a.feq_in[q] = t * (3.0 * (0.0 - a.p_shift) + (ref_flow ? 0.0 : br));
      a.enc.inlet_g[q] = static_cast<float>(a.feq_in[q] * static_cast<double>(a.enc.scale[q]));
    }
  }
  in.buf[0] = buf0;
  in.buf[1] = buf1;
  in.rec[0] = rec0;
  in.rec[1] = rec1;
  in.prev = prev;
  sl.bx_log2 = bx_log2_for(d->nx, d->tile_bx);
  in.bx_log2 = sl.bx_log2;
  in.parity0 = static_cast<int>(e->gstep & 1);
  // x-pairs: the 2-byte formats, and FP32 for the vortex (the FP32 cavity
  // measured faster in the engine with two cells of a column a thread)
  in.x2 = d->nx % 2 == 0 && (storage == IMEXLB_F16 || storage == IMEXLB_BF16 ||
                             (storage == IMEXLB_F32 && d->kase == IMEXLB_TGV));
  // rows staged in shared memory where they fit a stage (and tile_bx asks
  // for no register-staged tile width)
  in.staged = instance_staged(storage, d, sl.L, &in.geo) ? 1 : 0;
  if (in.staged) {
    in.tw = d->nx;
    in.th = in.geo.R;
  } else {
    const int bx = 1 << sl.bx_log2;
    in.th = (256 / bx) * (in.x2 ? (storage == IMEXLB_F32 ? 1 : 2) : cpt_of(storage));
    in.tw = bx * (in.x2 ? 2 : 1);
  }
  LaunchCfg cfg{d->kase == IMEXLB_TGV ? Bc::Periodic : Bc::Standard, static_cast<Store>(storage), CaseRule::None,
                storage == IMEXLB_F64 && e->exact};
  IMX_ECUDA(launch_init_f(cfg, sl.L, buf0, buf1, mom, mom + n, mom + 2 * n, mom + 3 * n, a.p_shift, a.enc, e->stream));
  if (rec0) {
    IMX_ECUDA(launch_cavity_records(sl.L, buf0, rec0, e->stream));
    IMX_ECUDA(launch_cavity_records(sl.L, buf1, rec1, e->stream));
  }
  std::memcpy(up + off_inst, &in, sizeof(EngInst));
  IMX_ECUDA(cudaMemcpyAsync(e->d_inst.p + s, up + off_inst, sizeof(EngInst), cudaMemcpyHostToDevice, e->stream));
  // no wait: the uploads follow the work already queued on the stream, and
  // the pinned buffer is reused once they are done
  IMX_ECUDA(e->staging.release_after(sb, e->stream));
  sl.used = true;
  e->slots[s] = sl;
  e->h_left[s] = ENG_NO_LIMIT;
  IMX_ECUDA(cudaMemcpyAsync(e->d_left.p + s, &e->h_left[s], sizeof(int), cudaMemcpyHostToDevice, e->stream));
  IMX_ECUDA(cudaMemsetAsync(e->d_taken.p + s, 0, sizeof(uint32_t), e->stream));
  e->dirty = true;
  *slot_out = s;
  return IMEXLB_OK;
}

int imexlb_engine_remove(imexlb_engine* e, int slot) {
  if (!e || slot < 0 || slot >= static_cast<int>(e->slots.size()) || !e->slots[slot].used)
    return efail(IMEXLB_E_ARG, "no such instance");
  IMX_ECUDA(cudaStreamSynchronize(e->stream));
  Slot& sl = e->slots[slot];
  e->arena.release(sl.off, sl.bytes);
  sl = Slot{};
  e->dirty = true;
  return IMEXLB_OK;
}

int imexlb_engine_limit(imexlb_engine* e, int slot, int steps) {
  if (!e || slot < 0 || slot >= static_cast<int>(e->slots.size()) || !e->slots[slot].used)
    return efail(IMEXLB_E_ARG, "no such instance");
  Slot& sl = e->slots[slot];
  EngInst& in = e->h_inst[slot];
  // an instance that stopped missed steps: realign its buffer parity with
  // the engine's (the next step reads the buffer of its run's parity).  The
  // updates follow the work already queued on the stream (the steps queued
  // before this call still see the old values), through a pinned staging
  // buffer, so the call does not wait for the GPU.
  const int parity0 = static_cast<int>((e->gstep ^ sl.run) & 1);
  const bool realign = parity0 != in.parity0;
  cudaError_t serr = cudaSuccess;
  const size_t inst_bytes = (sizeof(EngInst) + 15) & ~static_cast<size_t>(15);
  const int sb = e->staging.get(inst_bytes + sizeof(int), &serr);
  if (sb < 0) return efail(IMEXLB_E_NOMEM, std::string("pinned upload buffer: ") + cudaGetErrorString(serr));
  char* up = e->staging.ptr(sb);
  if (realign) {
    in.parity0 = parity0;
    std::memcpy(up, &in, sizeof(EngInst));
    IMX_ECUDA(cudaMemcpyAsync(e->d_inst.p + slot, up, sizeof(EngInst), cudaMemcpyHostToDevice, e->stream));
    e->dirty = true;  // the staged tiles' descriptors carry it too
  }
  e->h_left[slot] = steps < 0 ? ENG_NO_LIMIT : steps;
  std::memcpy(up + inst_bytes, &e->h_left[slot], sizeof(int));
  IMX_ECUDA(cudaMemcpyAsync(e->d_left.p + slot, up + inst_bytes, sizeof(int), cudaMemcpyHostToDevice, e->stream));
  IMX_ECUDA(e->staging.release_after(sb, e->stream));
  return IMEXLB_OK;
}

int imexlb_engine_step(imexlb_engine* e, int nsteps) {
  if (!e) return efail(IMEXLB_E_ARG, "null engine");
  if (nsteps < 0) return efail(IMEXLB_E_ARG, "negative step count");
  if (nsteps == 0) return IMEXLB_OK;
  int rc = rebuild_tiles(e);
  if (rc) return rc;
  int left = nsteps;
  while (left > 0) {
    const bool last = left == 1;
    if (!last && left >= 3 && (e->gstep & 1) == 0 && e->use_graph && !e->h_tiles.empty()) {
      if (!e->graph) {
        cudaGraph_t g = nullptr;
        IMX_ECUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t e1 = launch_engine(e, 0, 0);
        cudaError_t e2 = launch_engine(e, 1, 0);
        cudaError_t e3 = cudaStreamEndCapture(e->stream, &g);
        if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) {
          if (g) cudaGraphDestroy(g);
          return efail(IMEXLB_E_CUDA, "capturing the engine's step graph failed");
        }
        cudaError_t e4 = cudaGraphInstantiate(&e->graph, g, 0);
        cudaGraphDestroy(g);
        if (e4 != cudaSuccess) return efail(IMEXLB_E_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e4));
      }
      IMX_ECUDA(cudaGraphLaunch(e->graph, e->stream));
      e->gstep += 2;
      left -= 2;
      continue;
    }
    IMX_ECUDA(launch_engine(e, static_cast<int>(e->gstep & 1), last ? 1 : 0));
    ++e->gstep;
    --left;
  }
  for (size_t s = 0; s < e->slots.size(); ++s) {
    Slot& sl = e->slots[s];
    if (!sl.used) continue;
    int& left = e->h_left[s];
    const int done = left == ENG_NO_LIMIT ? nsteps : std::min(nsteps, left);
    if (left != ENG_NO_LIMIT) left -= done;
    sl.steps += done;
    sl.run += done;
  }
  return IMEXLB_OK;
}

int imexlb_engine_fields(imexlb_engine* e, int slot, double* u, double* v, double* w, double* p) {
  if (!e || slot < 0 || slot >= static_cast<int>(e->slots.size()) || !e->slots[slot].used)
    return efail(IMEXLB_E_ARG, "no such instance");
  const EngInst& in = e->h_inst[slot];
  const size_t n = static_cast<size_t>(e->slots[slot].ncell);
  double* dst[4] = {u, v, w, p};
  double* src[4] = {in.a.mu, in.a.mv, in.a.mw, in.a.mp};
  for (int c = 0; c < 4; ++c)
    if (dst[c]) IMX_ECUDA(cudaMemcpyAsync(dst[c], src[c], n * 8, cudaMemcpyDeviceToHost, e->stream));
  return sync_checked(e);
}

int imexlb_engine_plane(imexlb_engine* e, int slot, int k, double* u, double* v, double* w, double* p) {
  if (!e || slot < 0 || slot >= static_cast<int>(e->slots.size()) || !e->slots[slot].used)
    return efail(IMEXLB_E_ARG, "no such instance");
  const Slot& sl = e->slots[slot];
  if (k < 0 || k >= sl.d.nz) return efail(IMEXLB_E_ARG, "plane index outside the lattice");
  const EngInst& in = e->h_inst[slot];
  const size_t plane = static_cast<size_t>(sl.d.nx) * sl.d.ny;
  double* dst[4] = {u, v, w, p};
  double* src[4] = {in.a.mu, in.a.mv, in.a.mw, in.a.mp};
  for (int c = 0; c < 4; ++c)
    if (dst[c])
      IMX_ECUDA(cudaMemcpyAsync(dst[c], src[c] + plane * k, plane * 8, cudaMemcpyDeviceToHost, e->stream));
  return sync_checked(e);
}

int imexlb_engine_residuals(imexlb_engine* e, double* out, int n_out) {
  if (!e || !out) return efail(IMEXLB_E_ARG, "null argument");
  if (n_out < static_cast<int>(e->slots.size())) return efail(IMEXLB_E_ARG, "output shorter than max_instances");
  int rc = rebuild_tiles(e);
  if (rc) return rc;
  for (int s = 0; s < n_out; ++s) out[s] = NAN;
  if (e->h_tiles.empty()) return IMEXLB_OK;
  EngArgs ea{e->d_inst.p, e->d_tiles.p, e->d_stiles.p, e->d_left.p, static_cast<int>(e->h_tiles.size()), 0, 0,
              e->d_err.p};
  const int grid = std::min(e->grid * 2, ea.ntiles);
  engine_resid_kernel<<<grid, 256, 0, e->stream>>>(ea, e->d_part.p);
  const int ns = static_cast<int>(e->seg_slots.size());
  engine_resid_reduce<<<ns, 256, 0, e->stream>>>(e->d_seg.p, e->d_seg.p + ns, e->d_part.p, e->d_res.p);
  IMX_ECUDA(cudaGetLastError());
  std::vector<double> res(2 * static_cast<size_t>(ns));
  IMX_ECUDA(cudaMemcpyAsync(res.data(), e->d_res.p, res.size() * 8, cudaMemcpyDeviceToHost, e->stream));
  if (const int rc = sync_checked(e)) return rc;
  for (int g = 0; g < ns; ++g) {
    Slot& sl = e->slots[e->seg_slots[g]];
    const double d2 = res[2 * g], n2 = res[2 * g + 1];
    out[e->seg_slots[g]] = !sl.have_prev ? INFINITY : (n2 > 0 ? std::sqrt(d2 / n2) : (d2 > 0 ? INFINITY : 0.0));
    // -1: no step since the last check (stopped at its step limit), so no
    // change to measure -- not a converged solve
    if (sl.have_prev && sl.run == sl.run_checked) out[e->seg_slots[g]] = -1.0;
    // NaN: the velocity field is not finite (before the first check the
    // previous field is not yet defined, so only the current one counts)
    if (!std::isfinite(n2) || (sl.have_prev && !std::isfinite(d2))) out[e->seg_slots[g]] = NAN;
    sl.have_prev = true;
    sl.run_checked = sl.run;
  }
  return IMEXLB_OK;
}

int imexlb_engine_info(const imexlb_engine* e, imexlb_engine_stats* st) {
  if (!e || !st) return efail(IMEXLB_E_ARG, "null argument");
  st->instances = 0;
  st->cells = 0;
  for (const auto& sl : e->slots)
    if (sl.used) {
      ++st->instances;
      st->cells += sl.ncell;
    }
  st->budget_bytes = e->arena.size;
  st->used_bytes = e->arena.used;
  st->tiles = static_cast<int64_t>(e->h_tiles.size());
  st->steps = e->gstep;
  return IMEXLB_OK;
}

int imexlb_engine_instance_bytes(imexlb_storage storage, const imexlb_instance_desc* d, size_t* bytes) {
  if (!d || !bytes) return efail(IMEXLB_E_ARG, "null argument");
  const int elem = storage == IMEXLB_F64 ? 8 : (storage == IMEXLB_F32 ? 4 : 2);
  const Layout L = make_layout(d->nx, d->ny, d->nz, 0, elem);
  const int64_t n = static_cast<int64_t>(d->nx) * d->ny * d->nz;
  auto r = [](size_t x) { return (x + 511) & ~static_cast<size_t>(511); };
  const size_t mask = static_cast<size_t>((n + 255) & ~int64_t(255));
  *bytes = 2 * r(L.bytes()) + r(4 * n * 8) + r(3 * n * 8) + (d->kase == IMEXLB_SPHERE ? r(mask + 4 * n) : 0) +
           2 * record_bytes(storage, d, L);
  return IMEXLB_OK;
}

static CheckpointHeader instance_header(const imexlb_engine* e, const Slot& sl) {
  CheckpointHeader c{};
  std::memcpy(c.magic, "IMXLBCK1", 8);
  c.kind = 1;
  c.kase = sl.d.kase;
  c.storage = sl.storage;
  c.bc = IMEXLB_BC_STANDARD;
  c.nx = sl.d.nx;
  c.ny = sl.d.ny;
  c.nz = sl.d.nz;
  c.cur = 0;
  c.steps = sl.steps;
  c.buf_bytes = sl.L.bytes();
  c.nbuf = 1;
  c.mom_bytes = 4 * static_cast<uint64_t>(sl.ncell) * sizeof(double);
  c.tau0 = sl.d.tau0;
  return c;
}

int imexlb_engine_checkpoint_size(const imexlb_engine* e, int slot, size_t* bytes) {
  if (!e || !bytes || slot < 0 || slot >= static_cast<int>(e->slots.size()) || !e->slots[slot].used)
    return efail(IMEXLB_E_ARG, "no such instance");
  const Slot& sl = e->slots[slot];
  *bytes = sizeof(CheckpointHeader) + sl.L.bytes() + 4 * static_cast<size_t>(sl.ncell) * sizeof(double);
  return IMEXLB_OK;
}

int imexlb_engine_checkpoint_save(imexlb_engine* e, int slot, void* host, size_t bytes) {
  size_t need = 0;
  if (const int rc = imexlb_engine_checkpoint_size(e, slot, &need)) return rc;
  if (!host || bytes < need) return efail(IMEXLB_E_ARG, "checkpoint buffer too small (see imexlb_engine_checkpoint_size)");
  if (const int rc = sync_checked(e)) return rc;
  const Slot& sl = e->slots[slot];
  const EngInst& in = e->h_inst[slot];
  const int cur = static_cast<int>(sl.run & 1);  // the buffer the next step reads
  const CheckpointHeader c = instance_header(e, sl);
  char* p = static_cast<char*>(host);
  std::memcpy(p, &c, sizeof c);
  p += sizeof c;
  IMX_ECUDA(cudaMemcpyAsync(p, in.buf[cur], c.buf_bytes, cudaMemcpyDeviceToHost, e->stream));
  p += c.buf_bytes;
  IMX_ECUDA(cudaMemcpyAsync(p, in.a.mu, c.mom_bytes, cudaMemcpyDeviceToHost, e->stream));  // u, v, w, p contiguous
  IMX_ECUDA(cudaStreamSynchronize(e->stream));
  return IMEXLB_OK;
}

int imexlb_engine_restore(imexlb_engine* e, const imexlb_instance_desc* d, const void* host, size_t bytes,
                          int* slot_out) {
  if (!e || !d || !host || !slot_out) return efail(IMEXLB_E_ARG, "null argument");
  if (bytes < sizeof(CheckpointHeader)) return efail(IMEXLB_E_ARG, "not a checkpoint (too short)");
  CheckpointHeader c;
  std::memcpy(&c, host, sizeof c);
  if (std::memcmp(c.magic, "IMXLBCK1", 8) != 0 || c.kind != 1) return efail(IMEXLB_E_ARG, "not an engine checkpoint");
  if (c.kase != d->kase || c.storage < IMEXLB_F64 || c.storage > IMEXLB_BF16 || c.nx != d->nx || c.ny != d->ny ||
      c.nz != d->nz || c.tau0 != d->tau0 || c.nbuf != 1 || c.steps < 0)
    return efail(IMEXLB_E_ARG, "checkpoint belongs to an instance with other parameters");
  int slot = -1;
  if (const int rc = imexlb_engine_add_as(e, d, static_cast<imexlb_storage>(c.storage), &slot)) return rc;
  Slot& sl = e->slots[slot];
  const CheckpointHeader want = instance_header(e, sl);
  if (c.buf_bytes != want.buf_bytes || c.mom_bytes != want.mom_bytes ||
      bytes < sizeof c + c.buf_bytes + c.mom_bytes) {
    imexlb_engine_remove(e, slot);
    return efail(IMEXLB_E_ARG, "checkpoint truncated or of another layout");
  }
  EngInst& in = e->h_inst[slot];
  // at admission the next step reads buf[0] (parity0 = engine step parity)
  const char* p = static_cast<const char*>(host) + sizeof c;
  IMX_ECUDA(cudaMemcpyAsync(in.buf[0], p, c.buf_bytes, cudaMemcpyHostToDevice, e->stream));
  if (in.rec[0]) IMX_ECUDA(launch_cavity_records(sl.L, in.buf[0], in.rec[0], e->stream));
  p += c.buf_bytes;
  IMX_ECUDA(cudaMemcpyAsync(in.a.mu, p, c.mom_bytes, cudaMemcpyHostToDevice, e->stream));
  const uint32_t taken = static_cast<uint32_t>(c.steps);
  IMX_ECUDA(cudaMemcpyAsync(e->d_taken.p + slot, &taken, sizeof taken, cudaMemcpyHostToDevice, e->stream));
  IMX_ECUDA(cudaStreamSynchronize(e->stream));
  sl.steps = c.steps;
  sl.have_prev = false;
  *slot_out = slot;
  return IMEXLB_OK;
}

int imexlb_engine_synchronize(imexlb_engine* e) {
  if (!e) return efail(IMEXLB_E_ARG, "null engine");
  return sync_checked(e);
}

void imexlb_engine_destroy(imexlb_engine* e) {
  if (!e) return;
  cudaStreamSynchronize(e->stream);
  delete e;
}

}  // extern "C"
