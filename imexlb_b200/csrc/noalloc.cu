// Field reductions that allocate nothing.
//
// imexlb_reduce() keeps its block partial sums in device memory the lattice
// allocated with cudaMalloc.  Some callers cannot allocate at all: a host
// application that reserves all device memory up front and forbids later
// allocation (a server admitting work against a fixed HBM budget), code
// running where cudaMalloc's implicit synchronisation would stall a pipeline,
// or a plugin inside a framework that owns every device allocation.  For them,
// imexlb_reduce_fields_noalloc() runs the same two-pass reduction over
// caller-provided device fields with its partial sums in the fixed array
// below, and writes the result to a caller-provided device address.
//
// The array is a file-scope __device__ variable: every GPU that loads this
// library holds it (32 KiB) until the process exits.  Host code cannot use the
// array's name as a device address, so the first call on each device looks the
// address up with cudaGetSymbolAddress (with that device current) and keeps it
// together with the CUDA context it belongs to.  A reset of the device's
// primary context (cudaDeviceReset) reloads the module, and the array may then
// sit elsewhere: a call that finds a different current context looks the
// address up again.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/imexlb.h"
#include "lattice.h"

namespace {

constexpr int NA_THREADS = 256;
constexpr int64_t NA_CELLS_PER_BLOCK = 65536;  // each block reduces one contiguous chunk
constexpr int NA_MAX_PARTIALS = 4096;          // scratch capacity: one partial per block
constexpr int64_t NA_MAX_CELLS = NA_CELLS_PER_BLOCK * NA_MAX_PARTIALS;  // 268,435,456
constexpr int NA_MAX_DEVICES = 64;

__device__ __align__(256) double g_noalloc_partials[NA_MAX_PARTIALS];

// The maximum keeps a NaN (fmax would drop it), so a non-finite field shows
// in the result of every kind: sums turn NaN or infinite by themselves.
__device__ __forceinline__ double na_max(double a, double b) { return (a >= b || a != a) ? a : b; }

__device__ __forceinline__ double na_combine(int kind, double a, double b) {
  return kind == IMEXLB_REDUCE_UMAX ? na_max(a, b) : a + b;
}

__device__ __forceinline__ double na_block_reduce(int kind, double x) {
  __shared__ double sh[NA_THREADS / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x = na_combine(kind, x, __shfl_xor_sync(0xffffffffu, x, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = x;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x < 32) {
    r = threadIdx.x < NA_THREADS / 32 ? sh[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r = na_combine(kind, r, __shfl_xor_sync(0xffffffffu, r, o));
  }
  return r;
}

// Pass 1: block b reduces cells [b * 65536, min(n, (b + 1) * 65536)) and
// overwrites partial[b].  Every partial pass 2 reads is written by this call,
// so nothing in the scratch has to start at zero.
__global__ void na_pass1(int kind, const double* u, const double* v, const double* w, const double* p, int64_t n,
                         double* partial) {
  const int64_t begin = static_cast<int64_t>(blockIdx.x) * NA_CELLS_PER_BLOCK;
  const int64_t end = begin + NA_CELLS_PER_BLOCK < n ? begin + NA_CELLS_PER_BLOCK : n;
  double acc = 0.0;
  for (int64_t c = begin + threadIdx.x; c < end; c += NA_THREADS) {
    double x;
    if (kind == IMEXLB_REDUCE_MASS) {
      x = 3.0 * p[c];
    } else if (kind == IMEXLB_REDUCE_KINETIC) {
      x = 0.5 * (u[c] * u[c] + v[c] * v[c] + w[c] * w[c]);
    } else {
      x = sqrt(u[c] * u[c] + v[c] * v[c] + w[c] * w[c]);
    }
    acc = na_combine(kind, acc, x);
  }
  acc = na_block_reduce(kind, acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

__global__ void na_pass2(int kind, const double* partial, int nparts, double* out) {
  double acc = 0.0;
  for (int b = threadIdx.x; b < nparts; b += NA_THREADS) acc = na_combine(kind, acc, partial[b]);
  acc = na_block_reduce(kind, acc);
  if (threadIdx.x == 0) *out = acc;
}

std::mutex g_mu;
struct ScratchAddr {
  CUcontext ctx = nullptr;  // the context the address belongs to
  double* addr = nullptr;
};
ScratchAddr g_partials_addr[NA_MAX_DEVICES];

// cuCtxGetCurrent through the runtime's driver entry point (the library does
// not link the driver library directly); resolved once.
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
CtxGetCurrentFn ctx_get_current() {
  static CtxGetCurrentFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<CtxGetCurrentFn>(p);
  }();
  return fn;
}

// The device address of g_noalloc_partials on the current device: looked up
// on the first call on each device and again whenever the device's current
// context is no longer the one the address was looked up in.
int partials_on_current_device(double** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return imx::set_last_error(IMEXLB_E_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= NA_MAX_DEVICES) return imx::set_last_error(IMEXLB_E_UNSUPPORTED, "device ordinal above 63");
  const CtxGetCurrentFn get_ctx = ctx_get_current();
  if (!get_ctx) return imx::set_last_error(IMEXLB_E_CUDA, "no-alloc reduction: cuCtxGetCurrent is unavailable");
  CUcontext ctx = nullptr;
  if (get_ctx(&ctx) != CUDA_SUCCESS) ctx = nullptr;
  std::lock_guard<std::mutex> lock(g_mu);
  ScratchAddr& slot = g_partials_addr[dev];
  if (!slot.addr || !ctx || slot.ctx != ctx) {
    void* addr = nullptr;
    e = cudaGetSymbolAddress(&addr, g_noalloc_partials);  // makes the device's primary context current if none is
    if (e != cudaSuccess || !addr)
      return imx::set_last_error(IMEXLB_E_CUDA,
                                 std::string("cudaGetSymbolAddress(no-alloc scratch): ") + cudaGetErrorString(e));
    if (get_ctx(&ctx) != CUDA_SUCCESS) ctx = nullptr;
    slot.ctx = ctx;
    slot.addr = static_cast<double*>(addr);
  }
  *out = slot.addr;
  return IMEXLB_OK;
}

}  // namespace

extern "C" int imexlb_reduce_fields_noalloc(int kind, const double* u, const double* v, const double* w,
                                            const double* p, int64_t n, double* out, void* stream) {
  if (kind != IMEXLB_REDUCE_MASS && kind != IMEXLB_REDUCE_KINETIC && kind != IMEXLB_REDUCE_UMAX)
    return imx::set_last_error(IMEXLB_E_ARG, "no-alloc reduction: kind must be MASS, KINETIC or UMAX");
  if (!out) return imx::set_last_error(IMEXLB_E_ARG, "no-alloc reduction: null output address");
  if (kind == IMEXLB_REDUCE_MASS ? !p : (!u || !v || !w))
    return imx::set_last_error(IMEXLB_E_ARG, "no-alloc reduction: a field this reduction reads is null");
  if (n < 1) return imx::set_last_error(IMEXLB_E_ARG, "no-alloc reduction: n must be >= 1");
  if (n > NA_MAX_CELLS)
    return imx::set_last_error(IMEXLB_E_ARG, "no-alloc reduction: n = " + std::to_string(n) +
                                                 " exceeds the fixed scratch capacity of 268435456 cells");
  double* partial = nullptr;
  const int rc = partials_on_current_device(&partial);
  if (rc) return rc;
  const int nparts = static_cast<int>((n + NA_CELLS_PER_BLOCK - 1) / NA_CELLS_PER_BLOCK);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  na_pass1<<<nparts, NA_THREADS, 0, s>>>(kind, u, v, w, p, n, partial);
  na_pass2<<<1, NA_THREADS, 0, s>>>(kind, partial, nparts, out);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return imx::set_last_error(IMEXLB_E_CUDA, std::string("no-alloc reduction launch: ") + cudaGetErrorString(e));
  return IMEXLB_OK;
}
