// Shared-memory staged step for the 2-byte storage formats (FP16, BF16).
//
// The register-staged kernels keep every pulled population of a thread's
// cells in registers until it is used, so the bytes a warp can have in
// flight are bounded by its registers, and the step waits on DRAM latency
// long before it reaches DRAM bandwidth.  Here the loads are bulk
// asynchronous copies (cp.async.bulk, the untiled TMA path) into shared
// memory, completed on an mbarrier, so a block keeps the next tile in flight
// while it computes on the current one.
//
// A tile is R whole rows [j0, j0 + R) of plane k.  Population q of those
// cells pulls from rows j0 - e_y .. j0 + R - 1 - e_y of plane k - e_z,
// shifted by e_x along x.  The 2-byte layouts pad rows to 8 elements only,
// so those R source rows are one contiguous run of memory and a tile needs
// one bulk copy per population (two where a y wall or a periodic y cuts
// the run).  Whole rows also hold the x wrap of a periodic lattice.  A
// periodic y or z copies the wrapped rows; beyond a cavity wall the halfway
// bounce-back returns the cell's own opposite population, so the producer
// copies the tile's own rows of bb(q) into those slot rows.  Each copy
// costs the copy engine about the same whatever its size, so few large
// copies per tile are what keep DRAM busy.
//
// Warp 0 issues the copies of the block's tiles in order: tile i goes to
// stage i mod STAGES once all eight warps have released that stage's
// previous tile (its "empty" mbarrier), and the stage's "full" mbarrier
// counts the tile's bytes.  Every warp waits on "full", updates its cells
// and releases the stage.  Each thread updates x-pairs of cells with the
// same arithmetic as the register-staged x-pair kernels (finish_pair_row).
// The cavity's x-wall bounce-back values travel in wall records, one per
// row (WallRecord): the x-wall cells of a step write them (finish_pair_row),
// and the next step's tile copies the records of its rows with one more
// bulk copy, so no wall reads global memory here; only a sphere's solid
// links read the cell's own opposite population from global memory, in a
// second pass that only linked pairs take.
//
// Every wait on an mbarrier gives up after about a second of wall-clock time
// (%globaltimer), records the failure in the step's error word and leaves
// the kernel; the host reports it at its next synchronising call.
#pragma once

#include "step_core.cuh"

namespace imx {
namespace stage {

using namespace core;

constexpr int THREADS = 256;
constexpr int MAX_STAGES = 2;
constexpr int SLOT_CAP = 1024;                     // elements per population slot of a stage
constexpr int SLOT_UNITS = MAX_STAGES * SLOT_CAP;  // stages x elements per population slot
constexpr uint64_t WAIT_NS = 1000000000ull;

// Tile geometry of one lattice.  A tile is R whole rows of a plane, or (flat
// tiles) a run of C elements of a plane's rows taken as one line.
struct Geo {
  int P;       // staged row length: the layout's pitch (whole rows)
  int R;       // rows per tile (whole-row tiles)
  int cap;     // SLOT_CAP: R * P <= cap, or C + 2 FLAT_GUARD <= cap
  int stages;  // MAX_STAGES: stages * cap == SLOT_UNITS
  int nty;     // tiles per plane
  int flat;    // flat tiles (sphere channel)
  int C;       // elements per flat tile
};

// Flat tiles (the sphere channel: x not periodic, y and z periodic).  Whole
// rows of 768 elements make one-row tiles of 384 x-pairs for 256 threads, a
// quarter of whom then idle through a second pass.  A flat tile is the run
// [e0, e0 + C) of a plane's elements e = j P + x, across row ends; each
// population's slot holds the source run [e0 - e_y P - G, e0 + C - e_y P + G)
// of its plane (G = FLAT_GUARD elements a side, so that every pair's x - 1
// and x + 2 neighbours are staged, and 16-byte aligned), split in two where
// it wraps around the periodic y.  The pulled neighbour across a row end is
// never used: the inlet (x = 0) takes the inflow's equilibrium and the
// outlet (x = nx - 1) the cell's own column.
constexpr int FLAT_GUARD = 8;

// The 2-byte cavity's tiles also stage the wall records of their rows
// (WallRecord, 64 bytes a row) in an area of REC_ROWS records per stage.
constexpr int REC_ROWS = 16;
constexpr int REC_STAGE_BYTES = REC_ROWS * WallRecord::BYTES;

// Whole-row tiles for rows of `pitch` elements (a multiple of 8, so that
// every row starts on a 16-byte boundary; at most 1024): population slots
// of 1024 elements in 2 stages, at most `max_rows` rows a tile.  Fewer,
// larger copies beat deeper pipelines here (2 KB copies in 2 stages
// measured faster than 1 KB copies in 4 stages of the same shared memory).
inline bool make_geo(int ny, int64_t pitch, Geo* g, int max_rows = 1024) {
  if (pitch % 8 != 0 || pitch > 1024) return false;
  g->P = static_cast<int>(pitch);
  g->cap = SLOT_CAP;
  g->stages = MAX_STAGES;
  g->R = g->cap / g->P;
  if (g->R > max_rows) g->R = max_rows;
  if (g->R > ny) g->R = ny;
  g->nty = (ny + g->R - 1) / g->R;
  return true;
}

// Flat tiles of C = 1008 elements for a plane of ny rows of `pitch`
// elements, when the plane is long enough that a tile's source run wraps
// around y on one side at most.
inline bool make_geo_flat(int ny, int64_t pitch, Geo* g) {
  const int cap = SLOT_CAP, C = cap - 2 * FLAT_GUARD;
  const int64_t np = static_cast<int64_t>(ny) * pitch;
  if (pitch % 8 != 0 || np < C + 2 * pitch + 2 * FLAT_GUARD || np > (int64_t(1) << 30)) return false;
  g->P = static_cast<int>(pitch);
  g->R = 1;
  g->cap = cap;
  g->stages = MAX_STAGES;
  g->flat = 1;
  g->C = C;
  g->nty = static_cast<int>((np + C - 1) / C);
  return true;
}

// Tile geometry of the staged kernels for a lattice of nx x ny cells with
// rows of `pitch` elements, or false when it is not staged: nx even (the
// x-pairs); the cavity (wall records) at most REC_ROWS rows a tile and
// nx >= 4, so that a pair holds at most one x-wall cell; the sphere channel
// in flat tiles where its planes allow them.
inline bool staged_layout(CaseRule rule, int nx, int ny, int64_t pitch, Geo* g) {
  if (nx % 2 != 0) return false;
  g->flat = 0;
  g->C = 0;
  if (rule == CaseRule::SphereStd && nx >= 4 && make_geo_flat(ny, pitch, g)) return true;
  const bool rec = rule == CaseRule::CavityStd;
  if (rec && nx < 4) return false;
  return make_geo(ny, pitch, g, rec ? REC_ROWS : 1024);
}

// First row (whole-row tiles) or first element (flat tiles) of tile t of
// its plane, and its plane.
__host__ __device__ __forceinline__ int tile_origin(const Geo& g, int t) { return (t % g.nty) * (g.flat ? g.C : g.R); }
__host__ __device__ __forceinline__ int tile_plane(const Geo& g, int t) { return t / g.nty; }

// stages of 27 population slots, the wall-record areas (cavity), then the
// full and empty mbarriers
inline size_t smem_bytes(int elem, bool records) {
  return static_cast<size_t>(27) * SLOT_UNITS * elem + (records ? MAX_STAGES * REC_STAGE_BYTES : 0) +
         16 * MAX_STAGES;
}

// ------------------------------------------------------------ PTX helpers
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void bar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void bar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void bar_arrive_expect(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void bar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ bool bar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// try_wait that suspends at most about `hint_ns` (the instruction's own
// suspend-time hint) before it reports the phase as not yet complete.
// Non-blocking test of the phase of `parity` (mbarrier.test_wait).
__device__ __forceinline__ bool bar_test_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Below this a wait limit is finer than %globaltimer resolves: such a limit
// gives up after one failed poll.
constexpr uint64_t TIMER_FLOOR_NS = 1000;

// Wait for the phase of `parity` to complete; false after about limit_ns.
// A limit below a millisecond polls with the non-blocking test_wait, since
// one try_wait may suspend for longer than the limit.
__device__ __forceinline__ bool bar_wait_for(uint64_t* bar, uint32_t parity, uint64_t limit_ns) {
  if (limit_ns < 1000000ull) {
    const uint64_t t0 = global_ns();
    while (!bar_test_wait(bar, parity)) {
      if (limit_ns < TIMER_FLOOR_NS || global_ns() - t0 > limit_ns) return false;
    }
    return true;
  }
  if (bar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  while (true) {
    if (bar_try_wait(bar, parity)) return true;
    if (global_ns() - t0 > limit_ns) return false;
  }
}

// The same with the full bound of about a second.
__device__ __forceinline__ bool bar_wait(uint64_t* bar, uint32_t parity) { return bar_wait_for(bar, parity, WAIT_NS); }

// Bulk copy of `bytes` (a multiple of 16, both addresses 16-byte aligned)
// from global to this block's shared memory, completing on `bar`.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// e_y + 1 and e_z + 1 of population q, two bits each (q runtime)
constexpr uint64_t pack_axis(int axis) {
  uint64_t v = 0;
  for (int q = 0; q < Q; ++q) v |= static_cast<uint64_t>((axis == 1 ? D3Q27::ey[q] : D3Q27::ez[q]) + 1) << (2 * q);
  return v;
}
constexpr uint64_t EY_BITS = pack_axis(1), EZ_BITS = pack_axis(2);
__host__ __device__ __forceinline__ int ey_of(int q) { return static_cast<int>((EY_BITS >> (2 * q)) & 3u) - 1; }
__host__ __device__ __forceinline__ int ez_of(int q) { return static_cast<int>((EZ_BITS >> (2 * q)) & 3u) - 1; }

// The copies of population q for a tile: the source rows of tile rows
// [0, rv) as at most two contiguous runs, the second one a wrapped row
// (bytes 0 = no copy).
// the opposite population of q in the D3Q27 ordering (pairs 1-2, 3-4, ...)
__host__ __device__ constexpr int bb_of(int q) { return q == 0 ? 0 : ((q & 1) ? q + 1 : q - 1); }
constexpr bool bb_matches() {
  for (int q = 0; q < Q; ++q)
    if (bb_of(q) != D3Q27::bb[q]) return false;
  return true;
}
static_assert(bb_matches(), "bb_of follows the opposite table");

struct Run {
  int32_t src;  // element index within plane `pop`
  int32_t dst;  // element offset within the stage
  uint32_t bytes;
  int32_t pop;  // population whose plane the run reads
};

// Source rows that lie outside a periodic axis wrap around.  On a wall
// (WRAP_YZ false: the cavity) the halfway bounce-back returns the cell's own
// opposite population instead, so slot q's rows whose source is outside the
// box receive the tile's own rows of bb(q) (plane k, rows j0 + r), which the
// consumer reads unshifted.  Also compiled for the host, where
// imexlb_debug_stage_plan lists the copies for checks on the CPU.
template <bool WRAP_YZ, class A>
__host__ __device__ __forceinline__ void tile_runs(const A& a, const Geo& g, int q, int j0, int k, int rv, int elem,
                                          Run& main, Run& wrap) {
  main.bytes = 0;
  wrap.bytes = 0;
  main.pop = wrap.pop = q;
  const int32_t slot = q * SLOT_CAP;
  int kk = k - ez_of(q);
  if (kk < 0 || kk >= a.nz) {
    if (!WRAP_YZ) {
      // every row of the tile bounces: bb(q)'s own rows
      main.pop = bb_of(q);
      main.src = a.base32 + k * a.sz32 + j0 * a.pitch32;
      main.dst = slot;
      main.bytes = static_cast<uint32_t>(rv * g.P * elem);
      return;
    }
    kk = kk < 0 ? kk + a.nz : kk - a.nz;
  }
  const int y0 = j0 - ey_of(q);  // source row of tile row 0
  const int32_t plane = a.base32 + kk * a.sz32;
  const int r_lo = y0 < 0 ? -y0 : 0;
  const int r_hi = y0 + rv > a.ny ? a.ny - y0 : rv;
  main.src = plane + (y0 + r_lo) * a.pitch32;
  main.dst = slot + r_lo * g.P;
  main.bytes = r_hi > r_lo ? static_cast<uint32_t>((r_hi - r_lo) * g.P * elem) : 0u;
  // tile row 0 pulls from y = -1, or the last tile row from y = ny; |e_y| <= 1
  // allows one of them at most
  const bool first = r_lo > 0, last = r_hi < rv;
  if (WRAP_YZ) {
    wrap.src = plane + (first ? (a.ny - 1) * a.pitch32 : 0);  // the wrapped row
  } else {
    wrap.pop = bb_of(q);  // the tile's own row of bb(q)
    wrap.src = a.base32 + k * a.sz32 + (first ? j0 : j0 + rv - 1) * a.pitch32;
  }
  wrap.dst = slot + (first ? 0 : (rv - 1) * g.P);
  wrap.bytes = (first || last) ? static_cast<uint32_t>(g.P * elem) : 0u;
}

// The copies of population q for flat tile [e0, e0 + C) of plane k (the
// sphere channel, y and z periodic): the source run [e0 - e_y P - G,
// e0 + n - e_y P + G) of plane k - e_z, n = the tile's own length, as at most
// two runs, the second one the part that wraps around y.
template <class A>
__host__ __device__ __forceinline__ void tile_runs_flat(const A& a, const Geo& g, int q, int e0, int k, int elem,
                                                        Run& main, Run& wrap) {
  main.bytes = 0;
  wrap.bytes = 0;
  main.pop = wrap.pop = q;
  const int32_t np = a.ny * g.P;
  int kk = k - ez_of(q);
  kk = kk < 0 ? kk + a.nz : (kk >= a.nz ? kk - a.nz : kk);
  const int32_t plane = a.base32 + kk * a.sz32;
  const int n = np - e0 < g.C ? np - e0 : g.C;
  const int32_t s0 = e0 - ey_of(q) * g.P - FLAT_GUARD;  // source element of slot element 0
  const int32_t s1 = s0 + n + 2 * FLAT_GUARD;            // one past the last
  const int32_t slot = q * SLOT_CAP;
  if (s1 <= 0 || s0 >= np) {
    // the whole run lies across the y wrap (a short last tile of a plane)
    main.src = plane + (s1 <= 0 ? s0 + np : s0 - np);
    main.dst = slot;
    main.bytes = static_cast<uint32_t>((s1 - s0) * elem);
    return;
  }
  // the part inside [0, np), and the part below 0 or at np and above (the
  // run is shorter than the plane by two rows: never both)
  const int32_t lo = s0 < 0 ? 0 : s0, hi = s1 > np ? np : s1;
  main.src = plane + lo;
  main.dst = slot + (lo - s0);
  main.bytes = static_cast<uint32_t>((hi - lo) * elem);
  if (s0 < 0) {
    wrap.src = plane + (s0 + np);
    wrap.dst = slot;
    wrap.bytes = static_cast<uint32_t>(-s0 * elem);
  } else if (s1 > np) {
    wrap.src = plane;
    wrap.dst = slot + (np - s0);
    wrap.bytes = static_cast<uint32_t>((s1 - np) * elem);
  }
}

// The wall records of tile rows [j0, j0 + rv) of plane k: one contiguous
// run (element offset into the record buffer, bytes).
template <class A>
__host__ __device__ __forceinline__ void tile_records(const A& a, int j0, int k, int rv, int64_t& src,
                                                      uint32_t& bytes) {
  src = (static_cast<int64_t>(k) * a.ny + j0) * WallRecord::WORDS;
  bytes = static_cast<uint32_t>(rv * WallRecord::BYTES);
}

// Issue the copies of tile (j0, k) into stage `st` (called by a whole warp;
// lane q < 27 copies population q).  `src` is the buffer being read,
// population q at q * a.sq.  Lane 30 copies the tile's wall records from
// `rec_src` (a 2-byte cavity; null for none) to `rec_st`; lane 31 copies
// `xbytes` (a multiple of 16, 0 for none) from `xsrc` to `xdst`; all on the
// same mbarrier.  `a` is the lattice's StepArgs, or any type with its
// extent and addressing fields (nx, ny, nz, base32, sz32, pitch32, sq).
template <class T, bool WRAP_YZ, class A>
__device__ __forceinline__ void issue_tile(const A& a, const Geo& g, const T* src, int j0, int k, T* st,
                                           uint64_t* bar, const uint16_t* rec_src = nullptr,
                                           uint16_t* rec_st = nullptr, void* xdst = nullptr,
                                           const void* xsrc = nullptr, uint32_t xbytes = 0) {
  const int lane = threadIdx.x & 31;
  const int rv = a.ny - j0 < g.R ? a.ny - j0 : g.R;
  Run m{0, 0, 0u}, w{0, 0, 0u};
  if (lane < Q) {
    if (g.flat)
      tile_runs_flat(a, g, lane, j0, k, static_cast<int>(sizeof(T)), m, w);  // j0: the tile's first element
    else
      tile_runs<WRAP_YZ>(a, g, lane, j0, k, rv, static_cast<int>(sizeof(T)), m, w);
  }
  int64_t rsrc = 0;
  uint32_t rbytes = 0;
  if (lane == 30 && rec_src) tile_records(a, j0, k, rv, rsrc, rbytes);
  uint32_t total = m.bytes + w.bytes + rbytes + (lane == 31 ? xbytes : 0u);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) total += __shfl_xor_sync(0xffffffffu, total, o);
  if (lane == 0) bar_arrive_expect(bar, total);
  __syncwarp();
  if (m.bytes) bulk_g2s(st + m.dst, src + static_cast<int64_t>(m.pop) * a.sq + m.src, m.bytes, bar);
  if (w.bytes) bulk_g2s(st + w.dst, src + static_cast<int64_t>(w.pop) * a.sq + w.src, w.bytes, bar);
  if (rbytes) bulk_g2s(rec_st, rec_src + rsrc, rbytes, bar);
  if (lane == 31 && xbytes) bulk_g2s(xdst, xsrc, xbytes, bar);
}

// A stage that receives no copies: completes its full mbarrier at once
// (called by a whole warp, like issue_tile).
__device__ __forceinline__ void issue_skip(uint64_t* bar) {
  if ((threadIdx.x & 31) == 0) bar_arrive(bar);  // the phase's one arrival, no transactions
  __syncwarp();
}

// The x-pair (x, x + 1) in tile row r of tile (j0, k), read from the staged
// rows.  `st` is the stage as 4-byte words.  Reads only the fields of `a`
// before StepArgs::src.  EDGE = false promises that no boundary rule of the
// box applies to the pair but the cavity's x walls: for the cavity, no wall
// row or plane around it.  Cavity: `rec` is the stage's wall records (tile
// row r at r * WallRecord::WORDS), `rec_row` the pair's row in the record
// buffer this step writes.
template <Store S, Bc B, CaseRule RULE, bool EDGE, bool FLAT = false, bool SR = false, class P>
__device__ __forceinline__ void pair_from_stage(const StepArgs& a, const P& pl, const Geo& g, const uint32_t* st,
                                                const int x, const int r, const int j0, const int k,
                                                const bool store, const uint32_t seed, const uint16_t* rec = nullptr,
                                                uint16_t* rec_row = nullptr, const int flat_j = 0,
                                                const int flat_pw = 0) {
  // flat tiles: the pair's row and its word in the slot come from the caller
  const int j = FLAT ? flat_j : j0 + r;
  const int row = (r * g.P) >> 1;  // word offset of tile row r in a slot
  const int pw = FLAT ? flat_pw : row + (x >> 1);
  const bool left_edge = EDGE && x == 0, right_edge = EDGE && x + 2 >= a.nx;
  int lw, rw;  // the pairs holding x - 1 and x + 2
  if constexpr (FLAT) {
    // the guards hold both; across a row end their values go unused
    lw = pw - 1;
    rw = pw + 1;
  } else if constexpr (RULE == CaseRule::CavityStd) {
    // at an x wall the value comes from the wall record below; read the
    // pair's own word there, inside the row
    lw = row + ((x == 0 ? x : x - 2) >> 1);
    rw = row + ((x + 2 >= a.nx ? x : x + 2) >> 1);
  } else {
    lw = row + ((x == 0 ? a.nx - 2 : x - 2) >> 1);  // wrapped inside the row
    rw = row + ((x + 2 >= a.nx ? 0 : x + 2) >> 1);
  }
  constexpr int slotw = SLOT_CAP / 2;  // a compile-time stride: every slot read is [base + immediate]

  uint32_t raw[Q];
  static_for<0, Q>([&](auto qc) {
    constexpr int q = decltype(qc)::value;
    constexpr int ex = D3Q27::ex[q];
    const uint32_t* slot = st + q * slotw;
    const uint32_t pv = slot[pw];
    uint32_t v = pv;
    if constexpr (ex == 1) {
      v = pair_of(slot[lw] >> 16, pv);
    } else if constexpr (ex == -1) {
      uint32_t rlo = slot[rw] & 0xffffu;
      if constexpr (RULE == CaseRule::SphereStd) {
        if (right_edge) rlo = pv >> 16;  // zero-gradient outlet: the own column
      }
      v = pair_of(pv >> 16, rlo);
    }
    raw[q] = v;
  });

  const int32_t bself = a.base32 + k * a.sz32 + j * a.pitch32 + x;
  bool live0 = true, live1 = true;
  uint32_t links0 = 0, links1 = 0;  // sphere: solid-link bits of the two cells
  if constexpr (RULE == CaseRule::CavityStd) {
    // halfway bounce-back at the x walls: the cell's own opposite population
    // of the last step, from the row's wall record (x = 0: the lo side, for
    // e_x = +1; x = nx - 1: the hi side, for e_x = -1).  A y / z wall
    // crossed by the same link overrides it below with the same value.
    if (x == 0 || x + 2 >= a.nx) {
      const uint16_t* rr = rec + r * WallRecord::WORDS;
      const bool lo = x == 0;
      static_for<0, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        constexpr int ex = D3Q27::ex[q];
        if constexpr (ex != 0) {
          constexpr int m = WallRecord::slot(q);
          if constexpr (ex > 0) {
            if (lo) raw[q] = (raw[q] & 0xffff0000u) | rr[m];
          } else {
            if (!lo) raw[q] = (raw[q] & 0xffffu) | (static_cast<uint32_t>(rr[WallRecord::HI + m]) << 16);
          }
        }
      });
    }
  }
  if constexpr (RULE == CaseRule::CavityStd && EDGE) {
    uint32_t out_bits = 0;  // bit (3 dz + dy): source row outside the box
#pragma unroll
    for (int dz = 0; dz < 3; ++dz)
#pragma unroll
      for (int dy = 0; dy < 3; ++dy) {
        const int jj = j + dy - 1, kk = k + dz - 1;
        if (jj < 0 || jj >= a.ny || kk < 0 || kk >= a.nz) out_bits |= 1u << (3 * dz + dy);
      }
    if (out_bits) {
      // halfway bounce-back at the y and z walls: a link leaving the box
      // returns the cell's own opposite population, which the producer put
      // in slot q in place of the missing source row (tile_runs)
      static_for<0, Q>([&](auto qc) {
        constexpr int q = decltype(qc)::value;
        constexpr int ey = D3Q27::ey[q], ez = D3Q27::ez[q];
        if ((out_bits >> (3 * (1 - ez) + (1 - ey))) & 1u) raw[q] = st[q * slotw + pw];
      });
    }
  } else if constexpr (RULE == CaseRule::SphereStd) {
    // solid cells lie inside the box of linked cells: the sphere is enclosed
    // by the fluid cells whose links end in it
    const bool near = k >= a.near_lo[2] && k <= a.near_hi[2] && j >= a.near_lo[1] && j <= a.near_hi[1] &&
                      x + 1 >= a.near_lo[0] && x <= a.near_hi[0];
    if (near) {
      const int64_t cell = x + static_cast<int64_t>(a.nx) * (j + static_cast<int64_t>(a.ny) * k);
      links0 = a.links[cell];
      links1 = a.links[cell + 1];
      live0 = a.usr[cell] != 0;
      live1 = a.usr[cell + 1] != 0;
      if (links0 | links1) {
        static_for<0, Q>([&](auto qc) {
          constexpr int q = decltype(qc)::value;
          constexpr int qb = D3Q27::bb[q];
          const bool s0 = (links0 >> q) & 1u, s1 = (links1 >> q) & 1u;
          if (s0 || s1) {
            const uint32_t bbp = pl.load_pair(qb, bself);
            raw[q] = pair_of(s0 ? bbp : raw[q], s1 ? (bbp >> 16) : (raw[q] >> 16));
          }
        });
      }
    }
  }
  // the lid plane is a wall plane: only EDGE pairs can sit under it
  const bool lid = RULE == CaseRule::CavityStd && EDGE && k == a.nz - 1;
  finish_pair_row<S, RULE, RULE == CaseRule::CavityStd, SR>(a, pl, raw, x, j, k, lid, left_edge, live0, live1, store,
                                                            seed, links0, links1, rec_row);
}

// n / d for 0 <= n < 2048 and 8 <= 2 d <= 2048, without an integer division:
// (n + 1/2) / d lies at least 1/(2 d) >= 2^-11 from an integer, and the two
// round-to-nearest steps (the reciprocal and the product) move it by at most
// (n / d) 2^-23 <= 2^-14, so the truncation is the quotient.  `inv` is
// __frcp_rn(d).
__device__ __forceinline__ int small_quotient(int n, float inv) {
  return __float2int_rz((static_cast<float>(n) + 0.5f) * inv);
}

// The cells of tile (j0, k) from stage `st`, shared by the block's threads:
// thread slot p is the pair at x = 2 (p mod P/2) of tile row p div P/2, so
// a warp's pairs, and its stores, follow the rows' alignment in memory
// (mapping only the pairs inside the box, so that warps start mid-row,
// spread each warp's stores over more sectors and measured slower).
// Cavity pairs in a wall row or plane take the checked path (y / z
// bounce-back; a warp holds pairs of one or two rows, so the choice is
// nearly uniform across it).  Cavity: `rec` is the stage's wall records,
// `rec_out` the record buffer this step writes.
template <Store S, Bc B, CaseRule RULE, bool SR = false, class P>
__device__ __forceinline__ void consume_tile(const StepArgs& a, const P& pl, const Geo& g, const uint32_t* st,
                                             const int j0, const int k, const bool store, const uint32_t seed,
                                             const uint16_t* rec = nullptr, uint16_t* rec_out = nullptr) {
  const int rv = a.ny - j0 < g.R ? a.ny - j0 : g.R;
  const int half = g.P >> 1;
  const int npairs = g.R * half;  // at most SLOT_CAP / 2
  const float inv_half = __frcp_rn(static_cast<float>(half));
  if constexpr (RULE == CaseRule::CavityStd) {
    const bool wall_plane = k == 0 || k == a.nz - 1;
    uint16_t* const rec_tile = rec_out + (static_cast<int64_t>(k) * a.ny + j0) * WallRecord::WORDS;
    for (int p = threadIdx.x; p < npairs; p += THREADS) {
      const int r = small_quotient(p, inv_half), x = 2 * (p - r * half);
      if (r >= rv || x >= a.nx) continue;
      const int j = j0 + r;
      uint16_t* const rec_row = rec_tile + r * WallRecord::WORDS;
      if (wall_plane || j == 0 || j == a.ny - 1)
        pair_from_stage<S, B, RULE, true, false, SR>(a, pl, g, st, x, r, j0, k, store, seed, rec, rec_row);
      else
        pair_from_stage<S, B, RULE, false, false, SR>(a, pl, g, st, x, r, j0, k, store, seed, rec, rec_row);
    }
  } else if constexpr (RULE == CaseRule::SphereStd) {
    if (g.flat) {
      // flat tile [e0, e0 + n) (j0 holds e0): pair p is elements e0 + 2p and
      // e0 + 2p + 1, word p + G/2 of the slot
      const int e0 = j0;
      const int np = a.ny * g.P;
      const int n = np - e0 < g.C ? np - e0 : g.C;
      // row of element e0 + 2p: jb + (x0 + 2p) / P, x0 + 2p < P + C
      const int jb = e0 / g.P, x0 = e0 - jb * g.P;
      const float inv_p = __frcp_rn(static_cast<float>(g.P));
      for (int p = threadIdx.x; 2 * p < n; p += THREADS) {
        const int l = x0 + 2 * p, dj = small_quotient(l, inv_p);
        const int j = jb + dj, x = l - dj * g.P;
        if (x < a.nx)
          pair_from_stage<S, B, RULE, true, true, SR>(a, pl, g, st, x, 0, 0, k, store, seed, nullptr, nullptr, j,
                                                  p + FLAT_GUARD / 2);
      }
    } else {
      for (int p = threadIdx.x; p < npairs; p += THREADS) {
        const int r = small_quotient(p, inv_half), x = 2 * (p - r * half);
        if (r < rv && x < a.nx) pair_from_stage<S, B, RULE, true, false, SR>(a, pl, g, st, x, r, j0, k, store, seed);
      }
    }
  } else {
    for (int p = threadIdx.x; p < npairs; p += THREADS) {
      const int r = small_quotient(p, inv_half), x = 2 * (p - r * half);
      if (r < rv && x < a.nx) pair_from_stage<S, B, RULE, true, false, SR>(a, pl, g, st, x, r, j0, k, store, seed);
    }
  }
}

}  // namespace stage
}  // namespace imx
