// Host runtime behind the C ABI (include/imexlb.h): parameter parsing,
// case set-up, device buffers, the step loop and the output paths.
//
// Case set-up follows the reference's Initialize (tgv/src/lbm.cpp:195-218,
// lid_driven_cavity/src/lbm.cpp:191-210, sphere/src/lbm.cpp:221-254): the
// macroscopic fields are computed here in FP64 with the same expressions (and
// the same libm), then the device writes f = feq into both buffers.  Host code
// in this file is compiled with -ffp-contract=off so every operation rounds
// as written.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "../../include/imexlb.h"
#include "lattice.h"

using namespace imx;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

#define IMX_CUDA(call)                                                                             \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess)                                                                         \
      return fail(IMEXLB_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));               \
  } while (0)

constexpr double PI_REF = 3.1415926;  // tgv/src/lbm.cpp:5, tgv/src/System.cpp:20-21

// splitmix64 (Steele, Lea, Flood, "Fast splittable pseudorandom number
// generators", OOPSLA 2014): the sphere's `ran` field when the caller gives
// none.  ran(i, j, k) = mix(seed ^ index) % 100, independent of thread order.
uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}

// Device memory of single lattices comes from one stream-ordered pool per
// device that keeps freed memory reserved (up to POOL_KEEP_BYTES, or until
// imexlb_release_cached_memory), so that creating a lattice after another was
// destroyed neither maps new memory nor waits for the device, as cudaMalloc
// and cudaFree of a few hundred MB do (tens of ms for a 128^3 FP64 lattice).
constexpr uint64_t POOL_KEEP_BYTES = 16ull << 30;
constexpr int POOL_MAX_DEVICES = 64;
std::mutex g_pool_mu;
cudaMemPool_t g_pools[POOL_MAX_DEVICES] = {};

cudaError_t lattice_pool(cudaMemPool_t* out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= POOL_MAX_DEVICES) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_pool_mu);
  if (!g_pools[dev]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    if ((e = cudaMemPoolCreate(&pool, &props)) != cudaSuccess) return e;
    uint64_t keep = POOL_KEEP_BYTES;
    if ((e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess) return e;
    g_pools[dev] = pool;
  }
  *out = g_pools[dev];
  return cudaSuccess;
}

// A device array of a lattice, allocated from the lattice pool in the order
// of the lattice's stream and returned to it the same way.  alloc() waits
// for the stream once, so the memory is then usable from any stream and by
// synchronous copies.
template <class T>
struct DevArray {
  T* p = nullptr;
  size_t n = 0;
  cudaStream_t s = nullptr;
  ~DevArray() { reset(); }
  void reset() {
    if (p) cudaFreeAsync(p, s);
    p = nullptr;
    n = 0;
  }
  cudaError_t alloc(size_t count, cudaStream_t stream) {
    reset();
    if (!count) return cudaSuccess;
    cudaMemPool_t pool = nullptr;
    cudaError_t e = lattice_pool(&pool);
    if (e != cudaSuccess) return e;
    if ((e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&p), count * sizeof(T), pool, stream)) != cudaSuccess) {
      p = nullptr;
      return e;
    }
    n = count;
    s = stream;
    return cudaStreamSynchronize(stream);
  }
};

}  // namespace

namespace imx {
int set_last_error(int code, const std::string& msg) { return fail(code, msg); }

void set_reference_flow(Encoding& enc, double u, double omega) {
  enc.u_ref[0] = static_cast<float>(u);
  enc.u_ref[1] = enc.u_ref[2] = 0.f;
  const float om_u = static_cast<float>(omega) * enc.unit;  // as the kernels form it
  for (int q = 0; q < Q; ++q) {
    const double e = D3Q27::ex[q] * u;
    enc.br_ref[q] = static_cast<float>(3.0 * e + 4.5 * e * e - 1.5 * u * u);
    enc.kref[q] = -(om_u * enc.br_ref[q]);
  }
}

Layout make_layout(int nx, int ny, int nz, int g, int elem) {
  Layout L;
  L.nx = nx;
  L.ny = ny;
  L.nz = nz;
  L.g = g;
  L.elem = elem;
  L.ex = nx + 2 * g;
  L.ey = ny + 2 * g;
  L.ez = nz + 2 * g;
  // Rows start on 128-byte lines, except for the 2-byte formats without
  // ghosts: there a row is padded to 16 elements (one 32-byte sector) only,
  // so the rows of a plane are contiguous for nx a multiple of 16 and the
  // staged kernels copy several rows with one bulk copy.  (Rows padded to 8
  // elements, 16 bytes, start in mid-sector; the x-pair stores of a warp
  // then touch more sectors, and the 128^3 cavity ran 17 % slower.)
  const int64_t line = (elem == 2 && g == 0) ? 16 : 128 / elem;
  L.xoff = (line - (g % line)) % line;
  L.pitch = ((L.xoff + L.ex + line - 1) / line) * line;
  L.sz = L.pitch * L.ey;
  L.sq = L.sz * L.ez;
  return L;
}
}  // namespace imx

namespace imx {
// Standard sphere channel: bit q of a fluid cell's word is set when its pull
// along -e_q starts in a solid cell (y and z periodic; the x ends belong to
// the inlet and outlet rules).  lo/hi: bounding box of cells with a set bit.
// fn(k) for k in [0, nz), planes shared among host threads for large boxes
// (every plane is computed the same way whichever thread takes it)
template <class F>
static void for_planes(int nz, size_t plane_cells, F&& fn) {
  const unsigned hw = std::thread::hardware_concurrency();
  const int nt = static_cast<int>(std::min<size_t>(std::min(hw ? hw : 1u, 32u), nz * plane_cells / (1u << 18) + 1));
  if (nt <= 1) {
    for (int k = 0; k < nz; ++k) fn(k);
    return;
  }
  std::vector<std::thread> pool;
  for (int t = 0; t < nt; ++t)
    pool.emplace_back([&, t] {
      for (int k = t; k < nz; k += nt) fn(k);
    });
  for (auto& th : pool) th.join();
}

void solid_links(int nx, int ny, int nz, const uint8_t* fluid, std::vector<uint32_t>& links, int lo[3], int hi[3]) {
  const size_t plane = static_cast<size_t>(nx) * ny;
  links.assign(plane * nz, 0u);
  lo[0] = nx;
  lo[1] = ny;
  lo[2] = nz;
  hi[0] = hi[1] = hi[2] = -1;
  // the solid's box (per plane, then merged: each plane is one thread's)
  std::vector<int> pb(static_cast<size_t>(nz) * 6);
  for_planes(nz, plane, [&](int k) {
    int b[6] = {nx, ny, nz, -1, -1, -1};
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i)
        if (!fluid[i + static_cast<size_t>(nx) * j + plane * k]) {
          b[0] = std::min(b[0], i);
          b[1] = std::min(b[1], j);
          b[2] = std::min(b[2], k);
          b[3] = std::max(b[3], i);
          b[4] = std::max(b[4], j);
          b[5] = std::max(b[5], k);
        }
    std::copy(b, b + 6, pb.begin() + 6 * static_cast<size_t>(k));
  });
  int sb[6] = {nx, ny, nz, -1, -1, -1};
  for (int k = 0; k < nz; ++k)
    for (int d = 0; d < 3; ++d) {
      sb[d] = std::min(sb[d], pb[6 * static_cast<size_t>(k) + d]);
      sb[3 + d] = std::max(sb[3 + d], pb[6 * static_cast<size_t>(k) + 3 + d]);
    }
  if (sb[3] < 0) return;  // no solid
  // Only cells within one cell of the solid can link into it: that box,
  // or the whole axis where the solid reaches a periodic side (y, z) and
  // its neighbours wrap around.
  const int x0 = std::max(0, sb[0] - 1), x1 = std::min(nx - 1, sb[3] + 1);
  const bool ywrap = sb[1] == 0 || sb[4] == ny - 1, zwrap = sb[2] == 0 || sb[5] == nz - 1;
  const int y0 = ywrap ? 0 : sb[1] - 1, y1 = ywrap ? ny - 1 : sb[4] + 1;
  const int z0 = zwrap ? 0 : sb[2] - 1, z1 = zwrap ? nz - 1 : sb[5] + 1;
  std::vector<int> lb(static_cast<size_t>(nz) * 6);
  for_planes(nz, plane, [&](int k) {
    int b[6] = {nx, ny, nz, -1, -1, -1};
    if (k >= z0 && k <= z1) {
      const int ks[3] = {(k + 1) % nz, k, (k - 1 + nz) % nz};  // source plane for e_z = -1, 0, +1
      for (int j = y0; j <= y1; ++j) {
        const int js[3] = {(j + 1) % ny, j, (j - 1 + ny) % ny};
        for (int i = x0; i <= x1; ++i) {
          const size_t c = i + static_cast<size_t>(nx) * j + plane * k;
          if (!fluid[c]) continue;
          uint32_t bits = 0;
          for (int q = 0; q < Q; ++q) {
            const int si = i - D3Q27::ex[q];
            if (si < 0 || si >= nx) continue;
            const int sj = js[D3Q27::ey[q] + 1], sk = ks[D3Q27::ez[q] + 1];
            if (!fluid[si + static_cast<size_t>(nx) * sj + plane * sk]) bits |= 1u << q;
          }
          links[c] = bits;
          if (bits) {
            b[0] = std::min(b[0], i);
            b[1] = std::min(b[1], j);
            b[2] = std::min(b[2], k);
            b[3] = std::max(b[3], i);
            b[4] = std::max(b[4], j);
            b[5] = std::max(b[5], k);
          }
        }
      }
    }
    std::copy(b, b + 6, lb.begin() + 6 * static_cast<size_t>(k));
  });
  for (int k = 0; k < nz; ++k)
    for (int d = 0; d < 3; ++d) {
      lo[d] = std::min(lo[d], lb[6 * static_cast<size_t>(k) + d]);
      hi[d] = std::max(hi[d], lb[6 * static_cast<size_t>(k) + 3 + d]);
    }
}
}  // namespace imx

struct imexlb_lattice {
  imexlb_params P{};
  Layout L;
  LaunchCfg cfg{};
  DevArray<unsigned char> buf[2];
  DevArray<uint16_t> rec[2];  // wall records of buf[0], buf[1] (2-byte standard cavity, staged)
  int cur = 0;
  int64_t ncell = 0;
  DevArray<double> mom;       // u, v, w, p (4 * ncell)
  DevArray<double> prev_mom;  // u, v, w of the last residual call
  bool have_prev = false;
  DevArray<uint8_t> usr;      // interior mask (sphere)
  DevArray<uint32_t> links;   // standard sphere: per-cell solid-link bits
  DevArray<double> inlet;     // reference sphere inlet profile per z
  DevArray<int64_t> gtgt, gsrc;  // ghost-slot plan, 64-bit indices (very large buffers)
  DevArray<int2> gpk;            // the plan as packed 32-bit (target, source) pairs
  DevArray<int32_t> face_codes;  // reference cavity: the passes resolved per face-cell link
  int64_t gn = 0;
  DevArray<double> red;       // reduction partials + result
  DevArray<double> drag_part; // standard sphere: per-block drag partials of the last step
  int64_t drag_blocks = 0;
  DevArray<int> err;          // non-zero after a step kernel gave up waiting
  cudaStream_t stream = nullptr;
  int64_t steps = 0;
  std::vector<int32_t> usr_padded;  // host copy, padded box (reference sphere)
  std::vector<int32_t> ran;
  Encoding enc{};
  double p_shift = 0;
  StepArgs base_args;
  // per-launch timing: (start, end, kind) with kind 0 = step, 1 = ghost gather
  bool profiling = false;
  struct Timed {
    cudaEvent_t a, b;
    int kind;
  };
  std::vector<Timed> timed;
  std::vector<cudaEvent_t> event_pool;
  // asynchronous field reads (imexlb_get_fields_async): copies on their own
  // stream after `mom_ready`; the next moment-writing step waits `copy_done`
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t mom_ready = nullptr, copy_done = nullptr;
  bool copy_pending = false;
  ~imexlb_lattice() {
    if (copy_stream) {
      cudaStreamSynchronize(copy_stream);
      cudaStreamDestroy(copy_stream);
    }
    if (mom_ready) cudaEventDestroy(mom_ready);
    if (copy_done) cudaEventDestroy(copy_done);
    std::vector<cudaEvent_t> all(event_pool);
    for (auto& t : timed) {
      if (std::find(all.begin(), all.end(), t.a) == all.end()) all.push_back(t.a);
      if (std::find(all.begin(), all.end(), t.b) == all.end()) all.push_back(t.b);
    }
    for (auto e : all) cudaEventDestroy(e);
  }
  cudaEvent_t take_event() {
    if (!event_pool.empty()) {
      cudaEvent_t e = event_pool.back();
      event_pool.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
  }
};

namespace {

bool is_float_store(imexlb_storage s) { return s != IMEXLB_F64; }

// Macroscopic initial fields over the box the layout stores (padded box for
// reference boundaries, interior otherwise), x fastest.
void init_fields(imexlb_lattice* h, double* out) {
  case_fields(h->P, h->L, h->ran.empty() ? nullptr : h->ran.data(), &h->usr_padded, out);
}

}  // namespace

namespace imx {
void case_fields(const imexlb_params& P, const Layout& L, const int32_t* ran, std::vector<int32_t>* usr_padded,
                 double* out) {
  const size_t n = static_cast<size_t>(L.ex) * L.ey * L.ez;
  double* U = out;
  double* V = out + n;
  double* W = out + 2 * n;
  double* Pf = out + 3 * n;
  const int g = L.g;
  const int glx = P.nx, gly = P.ny, glz = P.nz;
  const size_t plane = static_cast<size_t>(L.ex) * L.ey;
  auto at = [&](int i, int j, int k) { return static_cast<size_t>(i) + L.ex * (static_cast<size_t>(j) + L.ey * k); };
  if (P.kase == IMEXLB_TGV) {
    // tgv/src/lbm.cpp:195-206 (cs2 = 1/3)
    const double u0 = P.u0, rho0 = P.rho0, cs2 = 1.0 / 3.0;
    for_planes(L.ez, plane, [&](int k) {
      for (int j = 0; j < L.ey; ++j)
        for (int i = 0; i < L.ex; ++i) {
          const double X = static_cast<double>(i - g) / static_cast<double>(glx) * 2.0 * PI_REF;
          const double Y = static_cast<double>(j - g) / static_cast<double>(gly) * 2.0 * PI_REF;
          const double Z = static_cast<double>(k - g) / static_cast<double>(glz) * 2.0 * PI_REF;
          const size_t c = at(i, j, k);
          U[c] = u0 * std::sin(X) * std::cos(Y) * std::cos(Z);
          V[c] = -u0 * std::cos(X) * std::sin(Y) * std::cos(Z);
          W[c] = 0;
          Pf[c] = rho0 * cs2 + rho0 * u0 * u0 / 16.0 * (std::cos(X * 2.0) + std::cos(Y * 2.0)) *
                                   (std::cos(Z * 2.0) + 2.0);
        }
    });
  } else if (P.kase == IMEXLB_SPHERE && P.bc == IMEXLB_BC_REFERENCE) {
    // sphere/src/lbm.cpp:231-242 over the padded box, with `ran` given
    const double u0 = P.u0;
    const int c8 = (glx - 1) / 8;
    const double r = (glx - 1) / 64.0;
    for_planes(L.ez, plane, [&](int k) {
      for (int j = 0; j < L.ey; ++j)
        for (int i = 0; i < L.ex; ++i) {
          const size_t c = at(i, j, k);
          const int dx = i - GHOST - c8, dy = j - GHOST - c8, dz = k - GHOST - c8;
          const double d2 = static_cast<double>(dx) * dx + static_cast<double>(dy) * dy + static_cast<double>(dz) * dz;
          const int s = (d2 <= r * r) ? 0 : 1;
          (*usr_padded)[c] = s;
          U[c] = (u0 * 4.0 * (k - GHOST) * (glz - 1 - (k - GHOST)) / (static_cast<double>(glz - 1) * (glz - 1))) * s *
                 (1.0 + ran[c] * 0.001);
          V[c] = W[c] = Pf[c] = 0.0;
        }
    });
  } else if (P.kase == IMEXLB_SPHERE) {
    // standard channel: uniform inlet velocity in the fluid at rest pressure
    const double ui = P.inlet_u;
    for_planes(L.ez, plane, [&](int k) {
      for (int j = 0; j < L.ey; ++j)
        for (int i = 0; i < L.ex; ++i) {
          const size_t c = at(i, j, k);
          const bool solid = std_sphere_solid(P, i, j, k);
          (*usr_padded)[c] = solid ? 0 : 1;
          U[c] = solid ? 0.0 : ui;
          V[c] = W[c] = Pf[c] = 0.0;
        }
    });
  } else {
    // cavity (both boundary kinds): u = p = 0 (lid_driven_cavity/src/lbm.cpp:191-198)
    for_planes(L.ez, plane, [&](int k) {
      for (int c4 = 0; c4 < 4; ++c4) std::memset(out + c4 * n + k * plane, 0, plane * sizeof(double));
    });
  }
}
}  // namespace imx

namespace imx {
bool std_sphere_solid(const imexlb_params& P, int i, int j, int k) {
  const double dx = i - P.sphere_c[0], dy = j - P.sphere_c[1], dz = k - P.sphere_c[2];
  return dx * dx + dy * dy + dz * dz <= 0.25 * P.sphere_d * P.sphere_d;
}

void std_sphere_mask(const imexlb_params& P, uint8_t* fluid) {
  const size_t plane = static_cast<size_t>(P.nx) * P.ny;
  for_planes(P.nz, plane, [&](int k) {
    for (int j = 0; j < P.ny; ++j)
      for (int i = 0; i < P.nx; ++i)
        fluid[i + static_cast<size_t>(P.nx) * j + plane * k] = std_sphere_solid(P, i, j, k) ? 0 : 1;
  });
}
}  // namespace imx

namespace {

// The cavity (at rest: u = p = 0, lid_driven_cavity/src/lbm.cpp:191-198, so
// f = feq(0, 0) = +0 in every storage format) and the standard sphere channel
// (inflow velocity in the fluid) have initial states the device builds from
// the case parameters and the mask; the vortex's and the reference sphere's
// initial fields are computed on the host with the reference's expressions
// and libm (tgv/src/lbm.cpp:195-206, sphere/src/lbm.cpp:231-242).
bool device_initial_state(const imexlb_params& P) {
  return P.kase == IMEXLB_CAVITY || (P.kase == IMEXLB_SPHERE && P.bc == IMEXLB_BC_STANDARD);
}

// The reference boundaries' ghost-slot gather into `dst`, previous-step
// values from `prev`, over whichever form of the plan the lattice holds.
cudaError_t ghost_gather(imexlb_lattice* h, void* dst, const void* prev) {
  if (h->gpk.p)
    return launch_ghost_gather_packed(h->cfg.store, dst, prev, h->gpk.p, h->gn, h->L.sq, h->enc, h->stream);
  return launch_ghost_gather(h->cfg.store, dst, prev, h->gtgt.p, h->gsrc.p, h->gn, h->L.sq, h->enc, h->stream);
}

int upload_device_case(imexlb_lattice* h) {
  const Layout& L = h->L;
  if (h->P.kase == IMEXLB_CAVITY) {
    IMX_CUDA(cudaMemsetAsync(h->buf[0].p, 0, h->buf[0].n, h->stream));
    IMX_CUDA(cudaMemsetAsync(h->buf[1].p, 0, h->buf[1].n, h->stream));
    IMX_CUDA(cudaMemsetAsync(h->mom.p, 0, h->mom.n * sizeof(double), h->stream));
  } else {
    // g = 0: the stored box is the interior, and init_f reads the moment views
    IMX_CUDA(cudaMemsetAsync(h->buf[0].p, 0, h->buf[0].n, h->stream));
    IMX_CUDA(cudaMemsetAsync(h->buf[1].p, 0, h->buf[1].n, h->stream));
    IMX_CUDA(launch_sphere_fields(h->usr.p, h->ncell, h->P.inlet_u, h->mom.p, h->stream));
    const double* src = h->mom.p;
    const int64_t n = h->ncell;
    IMX_CUDA(launch_init_f(h->cfg, L, h->buf[0].p, h->buf[1].p, src, src + n, src + 2 * n, src + 3 * n, h->p_shift,
                           h->enc, h->stream));
  }
  for (int b = 0; b < 2 && h->rec[b].p; ++b) IMX_CUDA(launch_cavity_records(L, h->buf[b].p, h->rec[b].p, h->stream));
  // reference boundaries: the first step's passes act on the initial state
  if (h->gn) IMX_CUDA(ghost_gather(h, h->buf[0].p, h->buf[1].p));
  IMX_CUDA(cudaStreamSynchronize(h->stream));
  h->cur = 0;
  h->steps = 0;
  h->have_prev = false;
  return IMEXLB_OK;
}

int upload_case(imexlb_lattice* h) {
  if (device_initial_state(h->P)) return upload_device_case(h);
  const Layout& L = h->L;
  const size_t n = static_cast<size_t>(L.ex) * L.ey * L.ez;
  std::unique_ptr<double[]> host(new double[4 * n]);  // every element written below
  init_fields(h, host.get());
  const double* U = host.get();
  const double* V = U + n;
  const double* W = U + 2 * n;
  const double* Pf = U + 3 * n;
  // Without ghosts the stored box is the interior: the fields go straight to
  // the moment views, which init_f reads.  With ghosts they go to a scratch
  // copy of the padded box and the interior is gathered on the host.
  const bool interior = L.g == 0;
  DevArray<double> tmp;
  if (!interior) IMX_CUDA(tmp.alloc(4 * n, h->stream));
  double* src = interior ? h->mom.p : tmp.p;
  IMX_CUDA(cudaMemcpyAsync(src, U, 4 * n * 8, cudaMemcpyHostToDevice, h->stream));
  IMX_CUDA(cudaMemsetAsync(h->buf[0].p, 0, h->buf[0].n, h->stream));
  IMX_CUDA(cudaMemsetAsync(h->buf[1].p, 0, h->buf[1].n, h->stream));
  IMX_CUDA(launch_init_f(h->cfg, L, h->buf[0].p, h->buf[1].p, src, src + n, src + 2 * n, src + 3 * n, h->p_shift,
                         h->enc, h->stream));
  for (int b = 0; b < 2 && h->rec[b].p; ++b) IMX_CUDA(launch_cavity_records(L, h->buf[b].p, h->rec[b].p, h->stream));
  if (!interior) {
    // the views after Initialize: interior moments
    std::vector<double> mom(4 * static_cast<size_t>(h->ncell));
    for (int k = 0; k < L.nz; ++k)
      for (int j = 0; j < L.ny; ++j)
        for (int i = 0; i < L.nx; ++i) {
          const size_t d = i + static_cast<size_t>(L.nx) * (j + static_cast<size_t>(L.ny) * k);
          const size_t c = (i + L.g) + static_cast<size_t>(L.ex) * ((j + L.g) + static_cast<size_t>(L.ey) * (k + L.g));
          mom[d] = U[c];
          mom[h->ncell + d] = V[c];
          mom[2 * h->ncell + d] = W[c];
          mom[3 * h->ncell + d] = Pf[c];
        }
    IMX_CUDA(cudaMemcpyAsync(h->mom.p, mom.data(), mom.size() * 8, cudaMemcpyHostToDevice, h->stream));
    IMX_CUDA(cudaStreamSynchronize(h->stream));  // before the host vector goes
  }
  // reference boundaries: the first step's passes act on the initial state
  if (h->gn) IMX_CUDA(ghost_gather(h, h->buf[0].p, h->buf[1].p));
  IMX_CUDA(cudaStreamSynchronize(h->stream));
  h->cur = 0;
  h->steps = 0;
  h->have_prev = false;
  return IMEXLB_OK;
}

// The face-code table of a reference cavity (FaceCodes in lattice.h) from
// its ghost-slot plan (tgt[n] takes src[n], encoded as in GhostPlan) in the
// index space of `slot(q, i, j, k)` (the pulled slot of interior cell (i, j, k)
// along -e_q): for every face cell, indexed by the first face it lies on, the
// source of each link whose pull leaves the box -- the plan's source when the
// pulled slot is planned, else the slot itself (never written: its initial
// value) -- and the links whose pulled slot a later step reads as its
// previous value.  False when an index does not fit 31 bits or a planned slot
// is not pulled by exactly one face cell (then the gather runs instead).
template <class Slot>
bool face_codes_generic(int nx, int ny, int nz, int64_t total, Slot slot, const std::vector<int64_t>& tgt,
                        const std::vector<int64_t>& src, std::vector<int32_t>& codes, int64_t base[6],
                        int32_t dim[6]) {
  if (total >= (int64_t(1) << 31) - 2) return false;
  std::unordered_map<int64_t, int64_t> plan;
  plan.reserve(tgt.size() * 2);
  std::unordered_set<int64_t> keep;  // slots read as previous values
  for (size_t n = 0; n < tgt.size(); ++n) {
    plan[tgt[n]] = src[n];
    if (src[n] <= -2) keep.insert(-src[n] - 2);
  }
  const int64_t cells[6] = {int64_t(ny) * nz, int64_t(ny) * nz, int64_t(nx) * nz,
                            int64_t(nx) * nz, int64_t(nx) * ny, int64_t(nx) * ny};
  int64_t off = 0;
  for (int f = 0; f < 6; ++f) {
    base[f] = off;
    dim[f] = f < 2 ? ny : nx;
    off += cells[f] * FACE_CODE_WORDS;
  }
  codes.assign(static_cast<size_t>(off), 0);
  size_t used = 0;
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const unsigned wf = (i == 0 ? 1u : 0u) | (i == nx - 1 ? 2u : 0u) | (j == 0 ? 4u : 0u) |
                            (j == ny - 1 ? 8u : 0u) | (k == 0 ? 16u : 0u) | (k == nz - 1 ? 32u : 0u);
        if (!wf) continue;
        int face = 0;
        while (!((wf >> face) & 1u)) ++face;
        const int fa = face < 2 ? j : i, fb = face < 4 ? k : j;
        int32_t* w = codes.data() + base[face] + (static_cast<int64_t>(fb) * dim[face] + fa) * FACE_CODE_WORDS;
        uint32_t keep_bits = 0;
        for (int q = 0; q < Q; ++q) {
          const int ex = D3Q27::ex[q], ey = D3Q27::ey[q], ez = D3Q27::ez[q];
          const bool leaves = (ex > 0 && (wf & 1u)) || (ex < 0 && (wf & 2u)) || (ey > 0 && (wf & 4u)) ||
                              (ey < 0 && (wf & 8u)) || (ez > 0 && (wf & 16u)) || (ez < 0 && (wf & 32u));
          if (!leaves) continue;
          const int64_t g = slot(q, i - ex, j - ey, k - ez);
          const auto it = plan.find(g);
          const int64_t code = it != plan.end() ? it->second : g;
          if (code >= total || code < -total - 2) return false;
          w[q] = static_cast<int32_t>(code);
          if (it != plan.end()) ++used;
          if (keep.count(g)) keep_bits |= 1u << q;
        }
        w[Q] = static_cast<int32_t>(keep_bits);
      }
  return used == tgt.size();  // every planned slot is some face cell's pulled slot
}

bool face_codes_for(const Layout& L, const std::vector<int64_t>& tgt, const std::vector<int64_t>& src,
                    std::vector<int32_t>& codes, int64_t base[6], int32_t dim[6]) {
  return face_codes_generic(L.nx, L.ny, L.nz, static_cast<int64_t>(L.sq) * Q,
                            [&](int q, int i, int j, int k) { return L.interior(q, i, j, k); }, tgt, src, codes, base,
                            dim);
}

// The device-side form of the reference boundary passes for one lattice
// shape: the ghost-slot plan in device indices, and for the cavity in FP64
// or FP32 storage the face-code table and face-cell list that replace it.
// It depends only on the case, the extents and the storage width (the
// reference sphere's mask is a function of the extents), so the last few
// are kept for the lattices created after them.
struct GhostSetup {
  int kase = 0, nx = 0, ny = 0, nz = 0, elem = 0;
  std::vector<int64_t> t, s;
  bool faces = false;
  std::vector<int32_t> codes, cells;
  int64_t base[6] = {};
  int32_t dim[6] = {};
};

std::mutex g_setup_mu;
std::vector<std::shared_ptr<const GhostSetup>> g_setups;  // most recent last
constexpr size_t SETUP_CACHE = 4;

std::shared_ptr<const GhostSetup> ghost_setup(const imexlb_params& P, const Layout& L, const int32_t* usr_padded,
                                              bool per_link, std::string* err) {
  {
    std::lock_guard<std::mutex> lock(g_setup_mu);
    for (const auto& g : g_setups)
      if (g->kase == P.kase && g->nx == P.nx && g->ny == P.ny && g->nz == P.nz && g->elem == L.elem &&
          g->faces == per_link)
        return g;
  }
  GhostPlan plan;
  if (!build_ghost_plan_keys(static_cast<int>(P.kase), P.nx, P.ny, P.nz, usr_padded, &plan, err)) return nullptr;
  auto g = std::make_shared<GhostSetup>();
  g->kase = P.kase;
  g->nx = P.nx;
  g->ny = P.ny;
  g->nz = P.nz;
  g->elem = L.elem;
  const int lx = P.nx + 2 * GHOST, ly = P.ny + 2 * GHOST;
  auto to_dev = [&](int64_t key) {
    const int q = static_cast<int>(key % Q);
    int64_t c = key / Q;
    const int i = static_cast<int>(c % lx);
    c /= lx;
    const int j = static_cast<int>(c % ly);
    const int k = static_cast<int>(c / ly);
    return L.idx(q, i, j, k);
  };
  g->t.resize(plan.tgt.size());
  g->s.resize(plan.src.size());
  for (size_t n = 0; n < g->t.size(); ++n) {
    g->t[n] = to_dev(plan.tgt[n]);
    const int64_t src = plan.src[n];
    g->s[n] = src >= 0 ? to_dev(src) : (src == -1 ? -1 : -to_dev(-src - 2) - 2);
  }
  // In target order the gather's stores run along the ghost rows of each
  // population plane, and their sources (mirror or shifted rows) with them;
  // the order of the copies does not matter (no target is a source of the
  // same step).
  {
    std::vector<int64_t> order(g->t.size());
    for (size_t n = 0; n < order.size(); ++n) order[n] = static_cast<int64_t>(n);
    std::sort(order.begin(), order.end(), [&](int64_t x, int64_t y) { return g->t[x] < g->t[y]; });
    std::vector<int64_t> t2(order.size()), s2(order.size());
    for (size_t n = 0; n < order.size(); ++n) {
      t2[n] = g->t[order[n]];
      s2[n] = g->s[order[n]];
    }
    g->t.swap(t2);
    g->s.swap(s2);
  }
  if (per_link) {
    if (!face_codes_for(L, g->t, g->s, g->codes, g->base, g->dim)) {
      if (err) *err = "the per-link form does not cover this lattice's boundary passes";
      return nullptr;
    }
    g->faces = true;
    for (int k = 0; k < P.nz; ++k)
      for (int j = 0; j < P.ny; ++j)
        for (int i = 0; i < P.nx; ++i)
          if (i == 0 || i == P.nx - 1 || j == 0 || j == P.ny - 1 || k == 0 || k == P.nz - 1)
            g->cells.push_back(i + P.nx * (j + P.ny * k));
  }
  std::lock_guard<std::mutex> lock(g_setup_mu);
  g_setups.push_back(g);
  if (g_setups.size() > SETUP_CACHE) g_setups.erase(g_setups.begin());
  return g;
}

}  // namespace

extern "C" {

void imexlb_params_default(imexlb_params* p) {
  std::memset(p, 0, sizeof(*p));
  p->kase = IMEXLB_TGV;
  p->bc = IMEXLB_BC_REFERENCE;
  p->storage = IMEXLB_F64;
  p->arith = IMEXLB_ARITH_EXACT;
  p->rho0 = 1.0;
  p->u0 = 0.05;
  p->seed = 5374857ULL;
}

int imexlb_system_read(const char* path, imexlb_case kase, imexlb_system* out) {
  if (!path || !out) return fail(IMEXLB_E_ARG, "null argument");
  std::ifstream in(path);
  if (!in) return fail(IMEXLB_E_IO, std::string("cannot open ") + path);
  imexlb_system s{};
  s.cs2 = 1.0 / 3.0;
  s.cs = std::sqrt(s.cs2);
  // tgv/src/System.cpp:12-15: three lines of whitespace-separated numbers;
  // Re, Time, inter, sx, sy, sz are integers
  in >> s.rho0 >> s.R >> s.Re;
  in >> s.u0 >> s.Time >> s.inter;
  in >> s.sx >> s.sy >> s.sz;
  if (!in) return fail(IMEXLB_E_IO, std::string("malformed input.in: ") + path);
  s.Ma = s.u0 / s.cs;
  if (kase == IMEXLB_TGV) {  // tgv/src/System.cpp:17-21
    s.Time = 100;
    s.inter = 10;
    s.miu = s.rho0 * s.u0 * s.sx / 2 / 3.1415926 / s.Re;
    s.tau = s.u0 * s.sx / s.Re / s.cs2 / 2 / 3.1415926;
  } else {  // lid_driven_cavity/src/System.cpp:17-19
    s.miu = s.rho0 * s.u0 * s.R / s.Re;
    s.tau = s.u0 * s.R / s.Re / s.cs2;
    if (kase == IMEXLB_SPHERE) {  // sphere/src/System.cpp:21-22
      s.Time = static_cast<int>(std::pow(2 * s.R, 2) / s.miu);
      s.inter = 1;
    }
  }
  *out = s;
  return IMEXLB_OK;
}

int imexlb_create(const imexlb_params* pin, imexlb_lattice** out) {
  if (!pin || !out) return fail(IMEXLB_E_ARG, "null argument");
  *out = nullptr;
  imexlb_params P = *pin;
  if (P.kase < IMEXLB_TGV || P.kase > IMEXLB_SPHERE) return fail(IMEXLB_E_ARG, "unknown case");
  if (P.bc != IMEXLB_BC_REFERENCE && P.bc != IMEXLB_BC_STANDARD && P.bc != IMEXLB_BC_SLAB &&
      P.bc != IMEXLB_BC_REFERENCE_LINKS)
    return fail(IMEXLB_E_ARG, "unknown boundary kind");
  if (P.bc == IMEXLB_BC_REFERENCE_LINKS &&
      (P.kase != IMEXLB_CAVITY || (P.storage != IMEXLB_F64 && P.storage != IMEXLB_F32)))
    return fail(IMEXLB_E_UNSUPPORTED, "per-link reference boundaries are for the cavity in FP64 or FP32 storage");
  const bool per_link = P.bc == IMEXLB_BC_REFERENCE_LINKS;
  const bool ref_bc = P.bc == IMEXLB_BC_REFERENCE || per_link;
  if (P.bc == IMEXLB_BC_SLAB && (P.kase != IMEXLB_CAVITY || (P.storage != IMEXLB_F64 && P.storage != IMEXLB_F32)))
    return fail(IMEXLB_E_UNSUPPORTED, "the slab boundaries are for the cavity in FP64 or FP32 storage");
  if (P.storage < IMEXLB_F64 || P.storage > IMEXLB_BF16) return fail(IMEXLB_E_ARG, "unknown storage");
  if (P.nx < 2 || P.ny < 2 || P.nz < 2) return fail(IMEXLB_E_ARG, "lattice extents must be >= 2");
  if (P.nz > 65535) return fail(IMEXLB_E_ARG, "nz above 65535");
  if (static_cast<double>(P.nx + 80) * (P.ny + 6) * (P.nz + 6) >= 2147483647.0)
    return fail(IMEXLB_E_ARG, "lattice too large: one population plane must stay below 2^31 values");
  if (!(P.tau0 > 0.0) || !std::isfinite(P.tau0)) return fail(IMEXLB_E_ARG, "tau0 must be positive");
  const bool ref_sphere = P.kase == IMEXLB_SPHERE && P.bc == IMEXLB_BC_REFERENCE;
  if (ref_sphere && (P.nx - 1) / 8 + (P.nx - 1) / 64.0 + 2 >= std::min(P.ny, P.nz))
    return fail(IMEXLB_E_ARG, "reference sphere (centre (nx-1)/8 on every axis) does not fit in ny, nz");
  if (P.kase == IMEXLB_CAVITY && !ref_bc && P.lid_u == 0.0) P.lid_u = P.u0;
  if (P.kase == IMEXLB_SPHERE && P.bc == IMEXLB_BC_STANDARD) {
    if (P.inlet_u == 0.0) P.inlet_u = P.u0;
    if (P.sphere_d == 0.0) P.sphere_d = P.nx / 24.0;
    if (P.sphere_c[0] == 0.0 && P.sphere_c[1] == 0.0 && P.sphere_c[2] == 0.0) {
      P.sphere_c[0] = P.nx / 4.0;
      P.sphere_c[1] = P.ny / 2.0;
      P.sphere_c[2] = P.nz / 2.0;
    }
  }

  std::unique_ptr<imexlb_lattice> h(new imexlb_lattice);
  h->P = P;
  h->P.ran = nullptr;
  h->stream = static_cast<cudaStream_t>(P.stream);
  const bool ghost = ref_bc && P.kase != IMEXLB_TGV;
  h->cfg.bc = P.kase == IMEXLB_TGV ? Bc::Periodic : (ghost ? Bc::Ghost : Bc::Standard);
  h->cfg.store = static_cast<Store>(P.storage);
  h->cfg.exact = P.storage == IMEXLB_F64 && P.arith == IMEXLB_ARITH_EXACT;
  if (P.kase == IMEXLB_TGV)
    h->cfg.rule = CaseRule::None;
  else if (P.kase == IMEXLB_CAVITY)
    h->cfg.rule = ghost ? CaseRule::CavityRef : (P.bc == IMEXLB_BC_SLAB ? CaseRule::SlabStd : CaseRule::CavityStd);
  else
    h->cfg.rule = ghost ? CaseRule::SphereRef : CaseRule::SphereStd;
  const int elem = P.storage == IMEXLB_F64 ? 8 : (P.storage == IMEXLB_F32 ? 4 : 2);
  h->L = make_layout(P.nx, P.ny, P.nz, ghost ? GHOST : 0, elem);
  const Layout& L = h->L;
  h->ncell = static_cast<int64_t>(P.nx) * P.ny * P.nz;

  // reduced precision: deviations from the rest state, scaled per population
  const double p_rest = P.kase == IMEXLB_TGV ? P.rho0 / 3.0 : 0.0;
  h->p_shift = is_float_store(P.storage) ? p_rest : 0.0;
  for (int q = 0; q < Q; ++q) {
    const double sc = store_scale(static_cast<Store>(P.storage), D3Q27::wclass[q]);
    h->enc.scale[q] = static_cast<float>(sc);
    h->enc.inv_scale[q] = static_cast<float>(1.0 / sc);
  }
  h->enc.unit = store_unit(static_cast<Store>(P.storage));
  h->enc.sr = stochastic_rounding_for(P.kase, P.storage);

  const size_t padded = static_cast<size_t>(L.ex) * L.ey * L.ez;
  if (P.kase == IMEXLB_SPHERE) {
    h->usr_padded.assign(padded, 1);
    if (ref_sphere) {
      h->ran.resize(padded);
      if (pin->ran) {
        std::memcpy(h->ran.data(), pin->ran, padded * sizeof(int32_t));
      } else {
        for (size_t c = 0; c < padded; ++c) h->ran[c] = static_cast<int32_t>(splitmix64(P.seed ^ c) % 100);
      }
    }
  }

  IMX_CUDA(h->buf[0].alloc(L.bytes(), h->stream));
  IMX_CUDA(h->buf[1].alloc(L.bytes(), h->stream));
  if (uses_wall_records(h->cfg, P.nx, P.ny, L.pitch))
    for (int b = 0; b < 2; ++b) IMX_CUDA(h->rec[b].alloc(static_cast<size_t>(P.ny) * P.nz * WallRecord::WORDS, h->stream));
  IMX_CUDA(h->mom.alloc(4 * static_cast<size_t>(h->ncell), h->stream));
  IMX_CUDA(h->red.alloc(2 * reduce_blocks() + 8, h->stream));
  // the residual's previous velocity field, allocated here so that a solve
  // loop's first residual check does not wait for the queued steps
  IMX_CUDA(h->prev_mom.alloc(3 * static_cast<size_t>(h->ncell), h->stream));
  IMX_CUDA(h->err.alloc(1, h->stream));
  IMX_CUDA(cudaMemset(h->err.p, 0, sizeof(int)));

  // base step arguments
  StepArgs& a = h->base_args;
  a.err = h->err.p;
  a.nx = P.nx;
  a.ny = P.ny;
  a.nz = P.nz;
  a.sq = L.sq;
  a.sz = L.sz;
  a.pitch = L.pitch;
  a.base = L.idx(0, L.g, L.g, L.g);
  for (int q = 0; q < Q; ++q) {
    a.off[q] = q * L.sq - (D3Q27::ez[q] * L.sz + D3Q27::ey[q] * L.pitch + D3Q27::ex[q]);
    a.rel[q] = static_cast<int32_t>(-(D3Q27::ez[q] * L.sz + D3Q27::ey[q] * L.pitch + D3Q27::ex[q]));
  }
  a.base32 = static_cast<int32_t>(a.base);
  a.sz32 = static_cast<int32_t>(L.sz);
  a.pitch32 = static_cast<int32_t>(L.pitch);
  a.tau_half = P.tau0 + 0.5;
  a.omega = 1.0 / (P.tau0 + 0.5);
  a.mu = h->mom.p;
  a.mv = h->mom.p + h->ncell;
  a.mw = h->mom.p + 2 * h->ncell;
  a.mp = h->mom.p + 3 * h->ncell;
  a.lid_u = h->cfg.rule == CaseRule::CavityRef ? 0.1 : P.lid_u;  // reference lid: literal 0.1
  a.rho_w = P.rho0;
  a.inlet_u = P.inlet_u;
  a.p_shift = h->p_shift;
  a.enc = h->enc;

  // the mask goes to the device before the initial state is set
  if (P.kase == IMEXLB_SPHERE) {
    std::vector<uint8_t> m(static_cast<size_t>(h->ncell));
    if (ref_sphere) {
      std::unique_ptr<double[]> fields(new double[4 * static_cast<size_t>(L.ex) * L.ey * L.ez]);
      init_fields(h.get(), fields.get());  // fills usr_padded
      for (int k = 0; k < P.nz; ++k)
        for (int j = 0; j < P.ny; ++j)
          for (int i = 0; i < P.nx; ++i)
            m[i + static_cast<size_t>(P.nx) * (j + static_cast<size_t>(P.ny) * k)] = static_cast<uint8_t>(
                h->usr_padded[(i + L.g) + static_cast<size_t>(L.ex) * ((j + L.g) + static_cast<size_t>(L.ey) * (k + L.g))]);
    } else {
      std_sphere_mask(P, m.data());  // the stored box is the interior (g = 0)
      for (size_t c = 0; c < m.size(); ++c) h->usr_padded[c] = m[c];
    }
    IMX_CUDA(h->usr.alloc(m.size(), h->stream));
    IMX_CUDA(cudaMemcpy(h->usr.p, m.data(), m.size(), cudaMemcpyHostToDevice));
    a.usr = h->usr.p;
    if (ref_sphere) {
      std::vector<double> prof(P.nz);
      const int glz = P.nz;
      for (int k = 0; k < P.nz; ++k)  // sphere/src/lbm.cpp:405
        prof[k] = P.u0 * 4.0 * k * (glz - 1 - k) / std::pow(static_cast<double>(glz - 1), 2);
      IMX_CUDA(h->inlet.alloc(prof.size(), h->stream));
      IMX_CUDA(cudaMemcpy(h->inlet.p, prof.data(), prof.size() * 8, cudaMemcpyHostToDevice));
      a.inlet = h->inlet.p;
    } else {
      std::vector<uint32_t> links;
      int lo[3], hi[3];
      solid_links(P.nx, P.ny, P.nz, m.data(), links, lo, hi);
      IMX_CUDA(h->links.alloc(links.size(), h->stream));
      IMX_CUDA(cudaMemcpy(h->links.p, links.data(), links.size() * 4, cudaMemcpyHostToDevice));
      a.links = h->links.p;
      for (int d = 0; d < 3; ++d) {
        a.near_lo[d] = lo[d];
        a.near_hi[d] = hi[d];
      }
      h->drag_blocks = step_grid_blocks(h->cfg, P.nx, P.ny, P.nz);
      IMX_CUDA(h->drag_part.alloc(3 * static_cast<size_t>(h->drag_blocks), h->stream));
      IMX_CUDA(cudaMemset(h->drag_part.p, 0, h->drag_part.n * sizeof(double)));
      // 2-byte x-pair formats store deviations from the inflow's equilibrium
      const double ui = P.inlet_u;
      const bool ref_flow = (P.storage == IMEXLB_F16 || P.storage == IMEXLB_BF16) && P.nx % 2 == 0;
      if (ref_flow) {
        set_reference_flow(h->enc, ui, 1.0 / (P.tau0 + 0.5));
        a.enc = h->enc;
      }
      // equilibrium populations of the inlet (deviation form)
      for (int q = 0; q < Q; ++q) {
        const double t = weight_of_class(D3Q27::wclass[q]);
        const double e = D3Q27::ex[q] * ui;
        // the reference's equilibrium bracket (tgv/src/lbm.cpp:228-232) of (ui, 0, 0): edu = e_x ui, udu = ui ui
        const double br = 3.0 * e + 4.5 * (e * e) - 1.5 * (ui * ui);
        a.feq_in[q] = t * (3.0 * (0.0 - h->p_shift) + (ref_flow ? 0.0 : br));
        a.enc.inlet_g[q] = static_cast<float>(a.feq_in[q] * static_cast<double>(a.enc.scale[q]));
      }
    }
  }

  if (ghost) {
    std::string err;
    const std::shared_ptr<const GhostSetup> g =
        ghost_setup(P, L, P.kase == IMEXLB_SPHERE ? h->usr_padded.data() : nullptr, per_link, &err);
    if (!g) return fail(IMEXLB_E_UNSUPPORTED, err);
    if (g->faces) {
      // the step kernel resolves the passes per link: no gather; its face
      // blocks take the face cells, listed plane by plane and row by row
      IMX_CUDA(h->face_codes.alloc(g->codes.size() + g->cells.size(), h->stream));
      IMX_CUDA(cudaMemcpy(h->face_codes.p, g->codes.data(), g->codes.size() * 4, cudaMemcpyHostToDevice));
      IMX_CUDA(cudaMemcpy(h->face_codes.p + g->codes.size(), g->cells.data(), g->cells.size() * 4,
                          cudaMemcpyHostToDevice));
      a.face_codes = h->face_codes.p;
      a.face_cells = h->face_codes.p + g->codes.size();
      a.n_face = static_cast<int32_t>(g->cells.size());
      for (int f = 0; f < 6; ++f) {
        a.face_base[f] = g->base[f];
        a.face_dim[f] = g->dim[f];
      }
    } else {
      h->gn = static_cast<int64_t>(g->t.size());
      const int64_t elems = static_cast<int64_t>(L.sq) * Q;
      if (elems < 2147483646ll) {
        // every index and source code fits 32 bits: one packed pair an entry
        std::vector<int2> pk(g->t.size());
        for (size_t n = 0; n < pk.size(); ++n)
          pk[n] = make_int2(static_cast<int32_t>(g->t[n]), static_cast<int32_t>(g->s[n]));
        IMX_CUDA(h->gpk.alloc(pk.size(), h->stream));
        IMX_CUDA(cudaMemcpy(h->gpk.p, pk.data(), pk.size() * sizeof(int2), cudaMemcpyHostToDevice));
      } else {
        IMX_CUDA(h->gtgt.alloc(g->t.size(), h->stream));
        IMX_CUDA(h->gsrc.alloc(g->s.size(), h->stream));
        IMX_CUDA(cudaMemcpy(h->gtgt.p, g->t.data(), g->t.size() * 8, cudaMemcpyHostToDevice));
        IMX_CUDA(cudaMemcpy(h->gsrc.p, g->s.data(), g->s.size() * 8, cudaMemcpyHostToDevice));
      }
    }
  }

  const int rc = upload_case(h.get());
  if (rc) return rc;
  *out = h.release();
  return IMEXLB_OK;
}

static int sync_checked(imexlb_lattice* h);

int imexlb_initialize(imexlb_lattice* h) {
  if (!h) return fail(IMEXLB_E_ARG, "null lattice");
  if (h->copy_pending)
    if (const int rc = sync_checked(h)) return rc;  // a field read still copies the moments
  return upload_case(h);
}

int imexlb_step(imexlb_lattice* h, int nsteps) {
  if (!h) return fail(IMEXLB_E_ARG, "null lattice");
  if (nsteps < 0) return fail(IMEXLB_E_ARG, "negative step count");
  StepArgs a = h->base_args;
  for (int s = 0; s < nsteps; ++s) {
    a.seed = sr_hash(static_cast<uint32_t>(h->steps));
    a.src = h->buf[h->cur].p;
    a.dst = h->buf[1 - h->cur].p;
    a.rec_src = h->rec[h->cur].p;
    a.rec_dst = h->rec[1 - h->cur].p;
    for (int q = 0; q < Q; ++q) {
      a.srcq[q] = h->buf[h->cur].p + static_cast<size_t>(q) * h->L.sq * h->L.elem;
      a.dstq[q] = h->buf[1 - h->cur].p + static_cast<size_t>(q) * h->L.sq * h->L.elem;
    }
    a.store = s == nsteps - 1;
    // the moments an asynchronous read is still copying are overwritten by
    // this call's last step only
    if (a.store && h->copy_pending) IMX_CUDA(cudaStreamWaitEvent(h->stream, h->copy_done, 0));
    const bool drag = a.store && h->drag_part.p;
    const bool drag_own = drag && drag_in_own_kernel(h->cfg.store);
    a.drag_part = (drag && !drag_own) ? h->drag_part.p : nullptr;
    imexlb_lattice::Timed t0{nullptr, nullptr, 0}, t1{nullptr, nullptr, 1};
    if (h->profiling) {
      t0.a = h->take_event();
      t0.b = h->take_event();
      IMX_CUDA(cudaEventRecord(t0.a, h->stream));
    }
    IMX_CUDA(launch_step(h->cfg, a, h->stream));
    if (h->profiling) {
      IMX_CUDA(cudaEventRecord(t0.b, h->stream));
      h->timed.push_back(t0);
    }
    if (drag_own) {
      StepArgs d = a;
      d.drag_part = h->drag_part.p;
      IMX_CUDA(launch_drag_links(h->cfg.store, d, h->stream));
    }
    if (h->gn) {
      if (h->profiling) {
        t1.a = t0.b;
        t1.b = h->take_event();
      }
      IMX_CUDA(ghost_gather(h, h->buf[1 - h->cur].p, h->buf[h->cur].p));
      if (h->profiling) {
        IMX_CUDA(cudaEventRecord(t1.b, h->stream));
        h->timed.push_back(t1);
      }
    }
    h->cur = 1 - h->cur;
    ++h->steps;
  }
  return IMEXLB_OK;
}

// Wait for the lattice's stream and report a step kernel that gave up
// waiting for its staged copies (its error word is then cleared).
static int sync_checked(imexlb_lattice* h) {
  if (h->copy_pending) {
    IMX_CUDA(cudaStreamSynchronize(h->copy_stream));
    h->copy_pending = false;
  }
  int word = 0;
  IMX_CUDA(cudaMemcpyAsync(&word, h->err.p, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  IMX_CUDA(cudaStreamSynchronize(h->stream));
  if (word) {
    IMX_CUDA(cudaMemset(h->err.p, 0, sizeof(int)));
    return fail(IMEXLB_E_CUDA, "a step kernel gave up waiting for its staged row copies; the lattice state is invalid");
  }
  return IMEXLB_OK;
}

int imexlb_get_fields(imexlb_lattice* h, double* u, double* v, double* w, double* p) {
  if (!h) return fail(IMEXLB_E_ARG, "null lattice");
  double* dst[4] = {u, v, w, p};
  for (int c = 0; c < 4; ++c)
    if (dst[c])
      IMX_CUDA(cudaMemcpyAsync(dst[c], h->mom.p + c * h->ncell, h->ncell * sizeof(double), cudaMemcpyDeviceToHost,
                               h->stream));
  return sync_checked(h);
}

int imexlb_get_fields_async(imexlb_lattice* h, double* u, double* v, double* w, double* p) {
  if (!h) return fail(IMEXLB_E_ARG, "null lattice");
  if (!h->copy_stream) {
    IMX_CUDA(cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking));
    IMX_CUDA(cudaEventCreateWithFlags(&h->mom_ready, cudaEventDisableTiming));
    IMX_CUDA(cudaEventCreateWithFlags(&h->copy_done, cudaEventDisableTiming));
  }
  IMX_CUDA(cudaEventRecord(h->mom_ready, h->stream));
  IMX_CUDA(cudaStreamWaitEvent(h->copy_stream, h->mom_ready, 0));
  double* dst[4] = {u, v, w, p};
  for (int c = 0; c < 4; ++c)
    if (dst[c])
      IMX_CUDA(cudaMemcpyAsync(dst[c], h->mom.p + c * h->ncell, h->ncell * sizeof(double), cudaMemcpyDeviceToHost,
                               h->copy_stream));
  IMX_CUDA(cudaEventRecord(h->copy_done, h->copy_stream));
  h->copy_pending = true;
  return IMEXLB_OK;
}

int imexlb_get_mask(imexlb_lattice* h, int32_t* usr) {
  if (!h || !usr) return fail(IMEXLB_E_ARG, "null argument");
  const Layout& L = h->L;
  for (int k = 0; k < L.nz; ++k)
    for (int j = 0; j < L.ny; ++j)
      for (int i = 0; i < L.nx; ++i) {
        const size_t d = i + static_cast<size_t>(L.nx) * (j + static_cast<size_t>(L.ny) * k);
        usr[d] = h->usr_padded.empty()
                     ? 1
                     : h->usr_padded[(i + L.g) + static_cast<size_t>(L.ex) * ((j + L.g) + static_cast<size_t>(L.ey) * (k + L.g))];
      }
  return IMEXLB_OK;
}

int imexlb_write_tecplot(imexlb_lattice* h, const char* path, int n) {
  if (!h || !path) return fail(IMEXLB_E_ARG, "null argument");
  const int64_t N = h->ncell;
  std::vector<double> f(4 * static_cast<size_t>(N));
  const int rc = imexlb_get_fields(h, f.data(), f.data() + N, f.data() + 2 * N, f.data() + 3 * N);
  if (rc) return rc;
  FILE* fp = std::fopen(path, "wb");
  if (!fp) return fail(IMEXLB_E_IO, std::string("cannot open ") + path);
  std::vector<unsigned char> hdr;
  auto put = [&](const void* x, size_t nb) {
    const unsigned char* c = static_cast<const unsigned char*>(x);
    hdr.insert(hdr.end(), c, c + nb);
  };
  auto I = [&](int32_t x) { put(&x, 4); };
  auto F = [&](float x) { put(&x, 4); };
  auto D = [&](double x) { put(&x, 8); };
  // header of tgv/src/lbm.cpp:467-647: magic, byte order, file type, title,
  // 7 variable names, zone "ZONE 001", solution time, ordered zone extents,
  // data section with FP64 variables and their min/max
  put("#!TDV112", 8);
  I(1);
  I(0);
  I(0);
  I(7);
  for (char c : std::string("xyzuvwp")) {
    I(c);
    I(0);
  }
  F(299.0f);
  for (char c : std::string("ZONE 001")) I(c);
  I(0);
  I(-1);
  D(static_cast<double>(n));
  I(0);
  I(-1);
  I(0);
  I(0);
  I(0);
  I(0);
  I(h->P.nx);
  I(h->P.ny);
  I(h->P.nz);
  I(0);
  F(357.0f);
  F(299.0f);
  for (int c = 0; c < 7; ++c) I(2);
  I(0);
  I(0);
  I(-1);
  for (int c = 0; c < 3; ++c) {
    D(0.0);
    D(1.0);
  }
  for (int c = 0; c < 4; ++c) {
    const double* a = f.data() + c * N;
    double mn = 1.7976931348623157e308, mx = -1.7976931348623157e308;
    for (int64_t e = 0; e < N; ++e) {
      if (a[e] > mx) mx = a[e];
      if (a[e] < mn) mn = a[e];
    }
    D(mn);
    D(mx);
  }
  bool ok = std::fwrite(hdr.data(), 1, hdr.size(), fp) == hdr.size();
  std::vector<double> coord(static_cast<size_t>(N));
  const int ext[3] = {h->P.nx, h->P.ny, h->P.nz};
  for (int axis = 0; axis < 3 && ok; ++axis) {
    for (int k = 0; k < h->P.nz; ++k)
      for (int j = 0; j < h->P.ny; ++j)
        for (int i = 0; i < h->P.nx; ++i) {
          const int c = axis == 0 ? i : (axis == 1 ? j : k);
          coord[i + static_cast<size_t>(h->P.nx) * (j + static_cast<size_t>(h->P.ny) * k)] =
              static_cast<double>(c) / (ext[axis] - 1);
        }
    ok = std::fwrite(coord.data(), 8, N, fp) == static_cast<size_t>(N);
  }
  if (ok) ok = std::fwrite(f.data(), 8, 4 * N, fp) == static_cast<size_t>(4 * N);
  if (std::fclose(fp) != 0 || !ok) return fail(IMEXLB_E_IO, std::string("write failed: ") + path);
  return IMEXLB_OK;
}

int imexlb_reduce(imexlb_lattice* h, int kind, double* out) {
  if (!h || !out) return fail(IMEXLB_E_ARG, "null argument");
  const int64_t N = h->ncell;
  const double* u = h->mom.p;
  const double* v = u + N;
  const double* w = u + 2 * N;
  const double* p = u + 3 * N;
  double* part = h->red.p;
  double* res = h->red.p + 2 * reduce_blocks();
  switch (kind) {
    case IMEXLB_REDUCE_MASS:
      IMX_CUDA(launch_reduce(RedKind::Mass, u, v, w, p, nullptr, nullptr, nullptr, N, part, res, h->stream));
      break;
    case IMEXLB_REDUCE_KINETIC:
      IMX_CUDA(launch_reduce(RedKind::Kinetic, u, v, w, p, nullptr, nullptr, nullptr, N, part, res, h->stream));
      break;
    case IMEXLB_REDUCE_UMAX:
      IMX_CUDA(launch_reduce(RedKind::UMax, u, v, w, p, nullptr, nullptr, nullptr, N, part, res, h->stream));
      break;
    case IMEXLB_REDUCE_RESIDUAL: {
      if (!h->prev_mom.p) IMX_CUDA(h->prev_mom.alloc(3 * static_cast<size_t>(N), h->stream));
      double nd[2] = {0.0, 0.0};
      if (h->have_prev) {
        IMX_CUDA(launch_residual_sums(u, v, w, h->prev_mom.p, h->prev_mom.p + N, h->prev_mom.p + 2 * N, N, part, res,
                                      h->stream));
        IMX_CUDA(cudaMemcpyAsync(nd, res, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
      }
      IMX_CUDA(cudaMemcpyAsync(h->prev_mom.p, u, 3 * N * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
      if (const int rc = sync_checked(h)) return rc;
      const double num = nd[0], den = nd[1];
      const bool first = !h->have_prev;
      h->have_prev = true;
      *out = first ? INFINITY : (den > 0 ? std::sqrt(num / den) : (num > 0 ? INFINITY : 0.0));
      if (!std::isfinite(num) || !std::isfinite(den))
        return fail(IMEXLB_E_STATE, "lattice is not finite (NaN/Inf in the velocity field)");
      return IMEXLB_OK;
    }
    case IMEXLB_REDUCE_DRAG: {
      if (!h->drag_part.p) return fail(IMEXLB_E_UNSUPPORTED, "drag needs the standard sphere channel");
      IMX_CUDA(launch_drag_sum(h->drag_part.p, h->drag_blocks, res, h->stream));
      IMX_CUDA(cudaMemcpyAsync(out, res, 3 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
      if (const int rc = sync_checked(h)) return rc;
      if (!std::isfinite(out[0]) || !std::isfinite(out[1]) || !std::isfinite(out[2]))
        return fail(IMEXLB_E_STATE, "drag is not finite");
      return IMEXLB_OK;
    }
    default:
      return fail(IMEXLB_E_ARG, "unknown or unsupported reduction");
  }
  IMX_CUDA(cudaMemcpyAsync(out, res, 8, cudaMemcpyDeviceToHost, h->stream));
  if (const int rc = sync_checked(h)) return rc;
  if (!std::isfinite(*out)) return fail(IMEXLB_E_STATE, "lattice is not finite (NaN/Inf in the moments)");
  return IMEXLB_OK;
}

int imexlb_reduce_async(imexlb_lattice* h, int kind, double* out) {
  if (!h || !out) return fail(IMEXLB_E_ARG, "null argument");
  const int64_t N = h->ncell;
  const double* u = h->mom.p;
  const double* v = u + N;
  const double* w = u + 2 * N;
  const double* p = u + 3 * N;
  double* part = h->red.p;
  double* res = h->red.p + 2 * reduce_blocks();  // res[0..1]: sums, res[2]: the residual
  double* val = res;
  switch (kind) {
    case IMEXLB_REDUCE_MASS:
      IMX_CUDA(launch_reduce(RedKind::Mass, u, v, w, p, nullptr, nullptr, nullptr, N, part, res, h->stream));
      break;
    case IMEXLB_REDUCE_KINETIC:
      IMX_CUDA(launch_reduce(RedKind::Kinetic, u, v, w, p, nullptr, nullptr, nullptr, N, part, res, h->stream));
      break;
    case IMEXLB_REDUCE_UMAX:
      IMX_CUDA(launch_reduce(RedKind::UMax, u, v, w, p, nullptr, nullptr, nullptr, N, part, res, h->stream));
      break;
    case IMEXLB_REDUCE_RESIDUAL:
      if (!h->prev_mom.p) IMX_CUDA(h->prev_mom.alloc(3 * static_cast<size_t>(N), h->stream));
      if (h->have_prev)
        IMX_CUDA(launch_residual_sums(u, v, w, h->prev_mom.p, h->prev_mom.p + N, h->prev_mom.p + 2 * N, N, part, res,
                                      h->stream));
      IMX_CUDA(launch_residual_finish(res, h->have_prev ? 0 : 1, res + 2, h->stream));
      IMX_CUDA(cudaMemcpyAsync(h->prev_mom.p, u, 3 * N * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
      h->have_prev = true;
      val = res + 2;
      break;
    default:
      return fail(IMEXLB_E_ARG, "unknown or unsupported asynchronous reduction");
  }
  IMX_CUDA(cudaMemcpyAsync(out, val, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  return IMEXLB_OK;
}

int imexlb_steps_taken(const imexlb_lattice* h, int64_t* steps) {
  if (!h || !steps) return fail(IMEXLB_E_ARG, "null argument");
  *steps = h->steps;
  return IMEXLB_OK;
}

int imexlb_footprint(const imexlb_lattice* h, size_t* device_bytes, double* bytes_per_cell_update) {
  if (!h) return fail(IMEXLB_E_ARG, "null lattice");
  if (device_bytes)
    *device_bytes = h->buf[0].n + h->buf[1].n + h->mom.n * 8 + h->prev_mom.n * 8 + h->usr.n + h->inlet.n * 8 +
                    h->gtgt.n * 8 + h->gsrc.n * 8 + h->gpk.n * 8 + h->face_codes.n * 4 + h->red.n * 8 + h->drag_part.n * 8 +
                    h->links.n * 4 +
                    (h->rec[0].n + h->rec[1].n) * sizeof(uint16_t);
  if (bytes_per_cell_update) *bytes_per_cell_update = 2.0 * Q * h->L.elem;
  return IMEXLB_OK;
}

int imexlb_ghost_plan(imexlb_case kase, int nx, int ny, int nz, const int32_t* usr_padded, int64_t* tgt,
                      int64_t* src, int64_t* n) {
  if (!n) return fail(IMEXLB_E_ARG, "null count");
  if (nx < 2 || ny < 2 || nz < 2) return fail(IMEXLB_E_ARG, "lattice extents must be >= 2");
  GhostPlan plan;
  std::string err;
  if (!build_ghost_plan_keys(static_cast<int>(kase), nx, ny, nz, usr_padded, &plan, &err))
    return fail(IMEXLB_E_UNSUPPORTED, err);
  const int64_t m = static_cast<int64_t>(plan.tgt.size());
  if (tgt && src) {
    if (*n < m) return fail(IMEXLB_E_ARG, "output arrays too small");
    std::memcpy(tgt, plan.tgt.data(), m * sizeof(int64_t));
    std::memcpy(src, plan.src.data(), m * sizeof(int64_t));
  }
  *n = m;
  return IMEXLB_OK;
}

int imexlb_profile(imexlb_lattice* h, int enable) {
  if (!h) return fail(IMEXLB_E_ARG, "null lattice");
  h->profiling = enable != 0;
  return IMEXLB_OK;
}

int imexlb_profile_read(imexlb_lattice* h, imexlb_kernel_times* out) {
  if (!h || !out) return fail(IMEXLB_E_ARG, "null argument");
  IMX_CUDA(cudaStreamSynchronize(h->stream));
  *out = imexlb_kernel_times{0.0, 0.0, 0, 0};
  std::vector<cudaEvent_t> done;
  for (auto& t : h->timed) {
    float ms = 0.f;
    IMX_CUDA(cudaEventElapsedTime(&ms, t.a, t.b));
    if (t.kind == 0) {
      out->step_ms += ms;
      ++out->step_launches;
    } else {
      out->ghost_ms += ms;
      ++out->ghost_launches;
    }
  }
  // a gather's start event is its step's end event: release each event once
  for (auto& t : h->timed) {
    if (std::find(done.begin(), done.end(), t.a) == done.end()) done.push_back(t.a);
    if (std::find(done.begin(), done.end(), t.b) == done.end()) done.push_back(t.b);
  }
  h->event_pool.insert(h->event_pool.end(), done.begin(), done.end());
  h->timed.clear();
  h->profiling = false;
  return IMEXLB_OK;
}

int imexlb_checkpoint_size(const imexlb_lattice* h, size_t* bytes) {
  if (!h || !bytes) return fail(IMEXLB_E_ARG, "null argument");
  *bytes = sizeof(CheckpointHeader) + h->buf[0].n + h->buf[1].n + h->mom.n * sizeof(double);
  return IMEXLB_OK;
}

static CheckpointHeader lattice_header(const imexlb_lattice* h) {
  CheckpointHeader c{};
  std::memcpy(c.magic, "IMXLBCK1", 8);
  c.kind = 0;
  c.kase = h->P.kase;
  c.storage = h->P.storage;
  c.bc = h->P.bc;
  c.nx = h->P.nx;
  c.ny = h->P.ny;
  c.nz = h->P.nz;
  c.cur = h->cur;
  c.steps = h->steps;
  c.buf_bytes = h->buf[0].n;
  c.nbuf = 2;
  c.mom_bytes = h->mom.n * sizeof(double);
  c.tau0 = h->P.tau0;
  return c;
}

int imexlb_checkpoint_save(imexlb_lattice* h, void* host, size_t bytes) {
  if (!h || !host) return fail(IMEXLB_E_ARG, "null argument");
  size_t need = 0;
  imexlb_checkpoint_size(h, &need);
  if (bytes < need) return fail(IMEXLB_E_ARG, "checkpoint buffer too small (see imexlb_checkpoint_size)");
  if (const int rc = sync_checked(h)) return rc;
  const CheckpointHeader c = lattice_header(h);
  char* p = static_cast<char*>(host);
  std::memcpy(p, &c, sizeof c);
  p += sizeof c;
  for (int b = 0; b < 2; ++b) {
    IMX_CUDA(cudaMemcpyAsync(p, h->buf[b].p, h->buf[b].n, cudaMemcpyDeviceToHost, h->stream));
    p += h->buf[b].n;
  }
  IMX_CUDA(cudaMemcpyAsync(p, h->mom.p, c.mom_bytes, cudaMemcpyDeviceToHost, h->stream));
  IMX_CUDA(cudaStreamSynchronize(h->stream));
  return IMEXLB_OK;
}

int imexlb_checkpoint_load(imexlb_lattice* h, const void* host, size_t bytes) {
  if (!h || !host) return fail(IMEXLB_E_ARG, "null argument");
  if (bytes < sizeof(CheckpointHeader)) return fail(IMEXLB_E_ARG, "not a checkpoint (too short)");
  CheckpointHeader c;
  std::memcpy(&c, host, sizeof c);
  const CheckpointHeader want = lattice_header(h);
  if (std::memcmp(c.magic, want.magic, 8) != 0 || c.kind != 0) return fail(IMEXLB_E_ARG, "not a lattice checkpoint");
  if (c.kase != want.kase || c.storage != want.storage || c.bc != want.bc || c.nx != want.nx || c.ny != want.ny ||
      c.nz != want.nz || c.buf_bytes != want.buf_bytes || c.nbuf != 2 || c.mom_bytes != want.mom_bytes ||
      c.tau0 != want.tau0 || (c.cur != 0 && c.cur != 1) || c.steps < 0)
    return fail(IMEXLB_E_ARG, "checkpoint belongs to a lattice with other parameters");
  size_t need = 0;
  imexlb_checkpoint_size(h, &need);
  if (bytes < need) return fail(IMEXLB_E_ARG, "checkpoint truncated");
  if (const int rc = sync_checked(h)) return rc;
  const char* p = static_cast<const char*>(host) + sizeof c;
  for (int b = 0; b < 2; ++b) {
    IMX_CUDA(cudaMemcpyAsync(h->buf[b].p, p, h->buf[b].n, cudaMemcpyHostToDevice, h->stream));
    p += h->buf[b].n;
  }
  IMX_CUDA(cudaMemcpyAsync(h->mom.p, p, c.mom_bytes, cudaMemcpyHostToDevice, h->stream));
  for (int b = 0; b < 2 && h->rec[b].p; ++b) IMX_CUDA(launch_cavity_records(h->L, h->buf[b].p, h->rec[b].p, h->stream));
  IMX_CUDA(cudaStreamSynchronize(h->stream));
  h->cur = c.cur;
  h->steps = c.steps;
  h->have_prev = false;
  return IMEXLB_OK;
}

int imexlb_synchronize(imexlb_lattice* h) {
  if (!h) return fail(IMEXLB_E_ARG, "null lattice");
  return sync_checked(h);
}

void imexlb_destroy(imexlb_lattice* h) {
  if (!h) return;
  cudaStreamSynchronize(h->stream);
  delete h;
}

int imexlb_set_wait_limit(imexlb_lattice* h, double seconds) {
  if (!h) return fail(IMEXLB_E_ARG, "null lattice");
  if (!(seconds > 0.0) || seconds > 1.0) return fail(IMEXLB_E_ARG, "wait limit must lie in (0, 1] seconds");
  const double ns = seconds * 1e9;
  h->base_args.wait_ns = ns < 1.0 ? 1ull : static_cast<uint64_t>(ns);
  return IMEXLB_OK;
}

int imexlb_set_rounding(imexlb_lattice* h, int stochastic) {
  if (!h) return fail(IMEXLB_E_ARG, "null lattice");
  if (stochastic != 0 && stochastic != 1) return fail(IMEXLB_E_ARG, "rounding must be 0 (nearest) or 1 (stochastic)");
  if (stochastic) {
    if (h->P.storage != IMEXLB_F16 && h->P.storage != IMEXLB_BF16)
      return fail(IMEXLB_E_UNSUPPORTED, "stochastic rounding is for the FP16 and BF16 storage formats");
    if (h->P.kase == IMEXLB_TGV) return fail(IMEXLB_E_UNSUPPORTED, "the vortex's kernels round to nearest only");
  }
  h->enc.sr = static_cast<uint32_t>(stochastic);
  h->base_args.enc.sr = h->enc.sr;
  return IMEXLB_OK;
}

int imexlb_release_cached_memory(void) {
  int dev = 0;
  IMX_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= POOL_MAX_DEVICES) return IMEXLB_OK;
  cudaMemPool_t pool = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_pool_mu);
    pool = g_pools[dev];
  }
  if (pool) {
    IMX_CUDA(cudaDeviceSynchronize());
    IMX_CUDA(cudaMemPoolTrimTo(pool, 0));
  }
  return IMEXLB_OK;
}

const char* imexlb_last_error(void) { return g_last_error.c_str(); }

const char* imexlb_version(void) { return "imexlb-b200 0.1 (sm_100a)"; }

// Not part of include/imexlb.h: the standard sphere's solid-link table of a
// fluid mask (x fastest), for checks on the CPU.  box: lo[3] then hi[3] of the
// linked cells (hi < 0: none).
int imexlb_debug_solid_links(int nx, int ny, int nz, const uint8_t* fluid, uint32_t* links, int32_t* box) {
  if (nx < 1 || ny < 1 || nz < 1 || !fluid || !links || !box) return IMEXLB_E_ARG;
  std::vector<uint32_t> l;
  int lo[3], hi[3];
  imx::solid_links(nx, ny, nz, fluid, l, lo, hi);
  std::copy(l.begin(), l.end(), links);
  for (int d = 0; d < 3; ++d) {
    box[d] = lo[d];
    box[3 + d] = hi[d];
  }
  return IMEXLB_OK;
}

// Not part of include/imexlb.h: the reference cavity's face-code table in the
// reference's slot keys (q + 27 (i + lx (j + ly k)) over the padded box), for
// a CPU restatement of the step that resolves the boundary passes per link.
// base_dim: the 6 face bases, then the 6 face widths.  Returns the number of
// words (call with codes = NULL to size), or -1 when the table is not used.
int64_t imexlb_debug_face_codes(int nx, int ny, int nz, int32_t* codes, int64_t max_words, int64_t* base_dim) {
  if (nx < 2 || ny < 2 || nz < 2) return -1;
  GhostPlan plan;
  std::string err;
  if (!build_ghost_plan_keys(IMEXLB_CAVITY, nx, ny, nz, nullptr, &plan, &err)) return -1;
  const int64_t lx = nx + 2 * GHOST, ly = ny + 2 * GHOST;
  auto key = [&](int q, int i, int j, int k) {
    return q + static_cast<int64_t>(Q) * ((i + GHOST) + lx * ((j + GHOST) + ly * (k + GHOST)));
  };
  std::vector<int32_t> c;
  int64_t base[6];
  int32_t dim[6];
  if (!face_codes_generic(nx, ny, nz, static_cast<int64_t>(Q) * lx * ly * (nz + 2 * GHOST), key, plan.tgt, plan.src, c,
                          base, dim))
    return -1;
  if (codes) {
    if (max_words < static_cast<int64_t>(c.size())) return -1;
    std::copy(c.begin(), c.end(), codes);
  }
  if (base_dim)
    for (int f = 0; f < 6; ++f) {
      base_dim[f] = base[f];
      base_dim[6 + f] = dim[f];
    }
  return static_cast<int64_t>(c.size());
}

// Not part of include/imexlb.h: lists the staged kernels' bulk copies so
// that their alignment and bounds are checked on the CPU (tests).  mode: 0
// cavity, 1 periodic vortex, 2 sphere channel; geo: 10 values (stage_plan).
int64_t imexlb_debug_stage_plan(int nx, int ny, int nz, int mode, int32_t* geo, int32_t* runs, int64_t max_runs) {
  return imx::stage_plan(nx, ny, nz, mode, geo, runs, max_runs);
}

}  // extern "C"
