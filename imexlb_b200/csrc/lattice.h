// Internal declarations shared by the host runtime (lattice.cu) and the
// device kernels (kernels.cu).  Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "d3q27.cuh"
#include "../../include/imexlb.h"

namespace imx {

enum class Bc : int { Periodic = 0, Ghost = 1, Standard = 2 };
enum class Store : int { F64 = 0, F32 = 1, F16 = 2, BF16 = 3 };
// Scale of a stored population of weight class `cls` (Encoding::scale):
// the FP16 format stores deviations times 2^14 / w_q, the BF16 format times
// 1 / w_q, FP32 and FP64 unscaled; the unit of the 2-byte collision is 2^14
// for FP16, else 1.  Compile-time values, so that the 2-byte step kernels
// take them as constants rather than loads.
IMX_HDC double store_scale(Store s, int cls) {
  return s == Store::F16 ? 16384.0 / weight_of_class(cls) : (s == Store::BF16 ? 1.0 / weight_of_class(cls) : 1.0);
}
IMX_HDC float store_unit(Store s) { return s == Store::F16 ? 16384.f : 1.f; }
// Which per-cell rules the step applies after the moments.
enum class CaseRule : int {
  None = 0,         // TGV
  CavityRef = 1,    // lid velocity forced on the top plane (Update)
  SphereRef = 2,    // solid mask times moments, inlet profile, outlet p = 0
  CavityStd = 3,    // moving-lid halfway bounce-back
  SphereStd = 4,    // channel: equilibrium inlet, zero-gradient outlet, solid sphere
  SlabStd = 5       // the cavity's bottom wall and moving lid, x and y periodic (plane Couette)
};

// Storage layout of one distribution buffer: 27 population planes, each a
// (z, y, x) box of stored extents (n + 2g) with x fastest.  Stored x = 0 sits
// `xoff` elements into its row so that interior x = 0 starts on a 128-byte
// boundary; rows, planes and populations are padded to 128 bytes (to 32
// bytes for the 2-byte formats without ghosts, see make_layout).
struct Layout {
  int nx = 0, ny = 0, nz = 0;  // interior
  int g = 0;                   // stored ghost width (3 for reference boundaries)
  int ex = 0, ey = 0, ez = 0;  // stored extents
  int64_t xoff = 0, pitch = 0, sz = 0, sq = 0;
  int elem = 8;  // bytes per stored value
  IMX_HD int64_t idx(int q, int i, int j, int k) const {  // stored coordinates
    return q * sq + k * sz + j * pitch + xoff + i;
  }
  IMX_HD int64_t interior(int q, int i, int j, int k) const { return idx(q, i + g, j + g, k + g); }
  size_t bytes() const { return static_cast<size_t>(sq) * Q * elem; }
};
Layout make_layout(int nx, int ny, int nz, int g, int elem);

// Per-population scaling of reduced-precision storage:
// stored = d_q * scale[q], d_q = stored * inv_scale[q], where d_q is the
// deviation f_q - 3 w_q p_shift.
// For the 2-byte formats scale[q] = unit / w_q, unit = 2^14 for FP16 (keeps
// small deviations out of the subnormals) and 1 for BF16; FP32 stores d_q.
// The standard sphere channel in the 2-byte x-pair formats measures the
// deviations from the equilibrium of the inflow instead of the rest state:
// d_q = f_q - w_q (3 p_shift + br_ref[q]), br_ref[q] = 3 c.u_ref + 4.5
// (c.u_ref)^2 - 1.5 |u_ref|^2 with u_ref the inlet velocity, so most of the
// channel stores small numbers; elsewhere u_ref = 0 and br_ref = 0.
struct Encoding {
  float scale[Q];
  float inv_scale[Q];
  float unit = 1.f;
  float u_ref[3] = {0.f, 0.f, 0.f};
  float br_ref[Q] = {};
  float kref[Q] = {};  // -omega unit br_ref[q], the collision's share of it
  uint32_t sr = 0;     // 2-byte formats: 1 = stochastic rounding of the stores
  // standard sphere, 2-byte pair kernels: StepArgs::feq_in[q] in stored
  // units, float(feq_in[q] * scale[q]) (the inlet column's values)
  float inlet_g[Q] = {};
};
// The stochastic-rounding hash: the 32-bit "lowbias32" integer finaliser
// (C. Wellons, hash-prospector, 2018).
IMX_HDC uint32_t sr_hash(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}
// Whether a lattice's 2-byte stores round stochastically (Encoding::sr):
// yes for the cavity and the sphere channel, driven flows that settle into
// a steady state, where round-to-nearest repeats the same error every step;
// no for the Taylor-Green vortex, a decaying flow without a steady state,
// whose error against FP64 is smaller with round-to-nearest (measured over
// 2000-16000 steps of 64^3 and 96^3 vortices).  `kase` is an imexlb_case,
// `storage` an imexlb_storage (2 = FP16, 3 = BF16).
inline uint32_t stochastic_rounding_for(int kase, int storage) {
  return (storage == 2 || storage == 3) && kase != 0 ? 1u : 0u;
}
// Set u_ref, br_ref and kref of `enc` for the reference velocity (u, 0, 0)
// and the relaxation rate omega.
void set_reference_flow(Encoding& enc, double u, double omega);

struct StepArgs {
  // Fields up to `src` are all that the shared-memory staged kernels read;
  // the engine copies this prefix (STAGED_ARGS_BYTES) into shared memory
  // with each tile.
  int nx = 0, ny = 0, nz = 0;
  int32_t base32 = 0, sz32 = 0, pitch32 = 0;
  int64_t sq = 0;
  double omega = 1;    // 1 / (tau0 + 0.5)
  double lid_u = 0;    // standard cavity lid speed; reference lid value
  double rho_w = 1;    // wall density of the moving-wall term
  double p_shift = 0;  // rest pressure removed from stored values (0 for FP64)
  double* mu = nullptr;
  double* mv = nullptr;
  double* mw = nullptr;
  double* mp = nullptr;
  const uint8_t* usr = nullptr;     // interior mask, 1 = fluid (sphere)
  const uint32_t* links = nullptr;  // standard sphere: per-cell bit q = the link along -e_q ends in the solid
  int near_lo[3] = {0, 0, 0};       // box of cells that have solid links
  int near_hi[3] = {-1, -1, -1};
  int store = 0;  // write moments this step
  uint32_t seed = 0;  // stochastic rounding: hash of the lattice's step count before this step
  Encoding enc;
  double feq_in[Q] = {};  // standard sphere: inlet equilibrium (deviation form)
  // ---- not read by the staged kernels
  const void* src = nullptr;
  void* dst = nullptr;
  const void* prev = nullptr;  // ghost gather: buffer of the previous step
  int64_t sz = 0, pitch = 0;
  int64_t base = 0;    // stored index of interior cell (0,0,0), population 0
  int64_t off[Q] = {}; // pull offset of population q relative to a cell's base index
  // plane addressing (step kernels): population q of a cell is
  // plane_q[base32 + k*sz32 + j*pitch32 + i], pulled from index + rel[q]
  const void* srcq[Q] = {};
  void* dstq[Q] = {};
  int32_t rel[Q] = {};
  double tau_half = 1; // tau0 + 0.5
  const double* inlet = nullptr; // per interior z: reference inlet velocity
  double inlet_u = 0;     // standard sphere inlet velocity
  double* drag_part = nullptr;  // standard sphere: per-block momentum-exchange partials (3 per block), or null
  int* err = nullptr;  // set non-zero by a kernel that gave up waiting (staged steps)
  // 2-byte standard cavity, staged kernels: the wall records of the buffer
  // read and of the buffer written (WallRecord)
  const uint16_t* rec_src = nullptr;
  uint16_t* rec_dst = nullptr;
  // Reference cavity with the boundary passes resolved in the step kernel
  // (FaceCodes): per face cell FACE_CODE_WORDS words, at
  // face_base[face] + (b * face_dim[face] + a) * FACE_CODE_WORDS; null: the
  // ghost-slot gather runs after each step instead
  const int32_t* face_codes = nullptr;
  int64_t face_base[6] = {};
  int32_t face_dim[6] = {};
  // its face cells (i + nx (j + ny k), in that order), which the first
  // face_layers z-layers of the step grid process, one cell a thread; the
  // other blocks leave face cells alone
  const int32_t* face_cells = nullptr;
  int32_t n_face = 0;
  int32_t face_layers = 0;
  // single-lattice staged kernels: bound on each wait for a tile's copies or
  // for a stage to be released (the drain of copies in flight after a block
  // gives up keeps the full second)
  uint64_t wait_ns = 1000000000ull;
};
// A face cell's words in the face-code table: word q (for a population whose
// pull leaves the box) names where the pulled value comes from --
//   code >= 0   element `code` of the buffer the step reads (this step's
//               post-collision value, or an unwritten ghost slot)
//   code == -1  zero
//   code <= -2  element (-code - 2) of the buffer the step writes (a ghost
//               slot as it stood after the previous step)
// -- and word 27 has bit q set when the step must also store that value in
// the pulled slot of the buffer it reads (a later step's "previous" value).
constexpr int FACE_CODE_WORDS = 28;
// Bytes of the StepArgs prefix the staged kernels read, rounded to 16.
constexpr size_t STAGED_ARGS_BYTES = (offsetof(StepArgs, src) + 15) & ~static_cast<size_t>(15);

// Ghost-slot plan for reference boundaries: after each step, slot tgt[n] of
// the new buffer receives the value named by src[n]:
//   src >= 0       the new buffer at index src (this step's post-collision)
//   src == -1      zero
//   src <= -2      the previous buffer at index (-src - 2)
struct GhostPlan {
  std::vector<int64_t> tgt, src;
};

// Build the plan in reference slot keys: key = q + 27*(i + lx*(j + ly*k)) over
// the padded box (lx = nx + 6).  Same encoding of src as GhostPlan.
// usr_padded: solid mask over the padded box (sphere), may be null.
// Returns false and sets *err if the passes would race.
bool build_ghost_plan_keys(int kase, int nx, int ny, int nz, const int32_t* usr_padded, GhostPlan* out,
                           std::string* err);

// Case set-up shared by single lattices and the engine: the initial u, v, w,
// p over the box the layout stores (x fastest) and, for spheres, the solid
// mask over the same box (reference: sphere/src/lbm.cpp:231-242; standard:
// the voxelised sphere |x - c|^2 <= d^2/4).  `ran` is the reference sphere's
// padded random field (unused otherwise).  `out` holds 4 n doubles, n the
// stored box's cells: u, then v, w, p; every element is written (the host's
// cores share the planes), so it may be uninitialised memory, such as a
// pinned upload buffer.  `usr_padded` (spheres) holds n values.
void case_fields(const imexlb_params& P, const Layout& L, const int32_t* ran, std::vector<int32_t>* usr_padded,
                 double* out);
// The standard sphere channel's voxelised sphere: cell (i, j, k) is solid
// when |x - c|^2 <= d^2 / 4 (each operation rounded on its own).
bool std_sphere_solid(const imexlb_params& P, int i, int j, int k);
// Its fluid mask (1 = fluid) over the interior, x fastest (ncell values).
void std_sphere_mask(const imexlb_params& P, uint8_t* fluid);
void solid_links(int nx, int ny, int nz, const uint8_t* fluid, std::vector<uint32_t>& links, int lo[3], int hi[3]);

// Header of a checkpoint (imexlb_checkpoint_*, imexlb_engine_checkpoint_*):
// the state follows it as nbuf distribution buffers of buf_bytes each, then
// the moments (mom_bytes).
struct CheckpointHeader {
  char magic[8];       // "IMXLBCK1"
  int32_t kind;        // 0 lattice, 1 engine instance
  int32_t kase, storage, bc;
  int32_t nx, ny, nz, cur;
  int64_t steps;
  uint64_t buf_bytes, nbuf, mom_bytes;
  double tau0;
  char pad[48];
};
static_assert(sizeof(CheckpointHeader) == 128, "checkpoint header layout");

// Record the calling thread's last error message (imexlb_last_error) and
// return `code`.
int set_last_error(int code, const std::string& msg);

// ---------------------------------------------------------------- launchers
struct LaunchCfg {
  Bc bc;
  Store store;
  CaseRule rule;
  bool exact;
};

// The staged kernels of this configuration keep wall records (WallRecord,
// one per row (j, k), ny * nz * WallRecord::BYTES bytes a buffer parity).
bool uses_wall_records(const LaunchCfg& c, int nx, int ny, int64_t pitch);
// Fill the wall records of distribution buffer `buf` (a 2-byte layout),
// after the buffer was written other than by a step.
cudaError_t launch_cavity_records(const Layout& L, const void* buf, uint16_t* rec, cudaStream_t s);
// Copy plan of the shared-memory staged kernels for a 2-byte lattice of
// nx x ny x nz: mode 0 the cavity (walls), 1 the periodic vortex, 2 the
// sphere channel (flat tiles where its planes allow them).  geo (10
// values): P, R, cap, nty, the layout's sq, sz, pitch and base, then flat
// and C.  runs: up to max_runs records (tile, q, population read, source
// element, stage element, bytes); the cavity's wall-record copy of a tile
// has q = Q, population -1 and its element offset in the record buffer.
// Returns the number of copies, or -1 when the lattice is not staged.
int64_t stage_plan(int nx, int ny, int nz, int mode, int32_t* geo, int32_t* runs, int64_t max_runs);
cudaError_t launch_init_f(const LaunchCfg& c, const Layout& L, void* buf0, void* buf1, const double* u,
                          const double* v, const double* w, const double* p, double p_shift, const Encoding& enc,
                          cudaStream_t s);
cudaError_t launch_step(const LaunchCfg& c, const StepArgs& a, cudaStream_t s);
// Initial u, v, w, p of the standard sphere channel from its interior fluid
// mask (out: 4 n values; the inflow velocity ui in the fluid, rest elsewhere).
cudaError_t launch_sphere_fields(const uint8_t* fluid, int64_t n, double ui, double* out, cudaStream_t s);
cudaError_t launch_ghost_gather(Store st, void* dst, const void* prev, const int64_t* tgt, const int64_t* src,
                                int64_t n, int64_t sq, const Encoding& enc, cudaStream_t s);
// The same with the plan packed as (target, source) 32-bit pairs, for
// buffers of fewer than 2^31 - 2 elements.
cudaError_t launch_ghost_gather_packed(Store st, void* dst, const void* prev, const int2* plan, int64_t n, int64_t sq,
                                       const Encoding& enc, cudaStream_t s);
dim3 step_block(int nx);
// Blocks that write one drag partial each: the step launch of this
// configuration, or the drag kernel's blocks for the 2-byte formats.
int64_t step_grid_blocks(const LaunchCfg& c, int nx, int ny, int nz);
cudaError_t launch_drag_sum(const double* part, int64_t nblk, double* out, cudaStream_t s);
// 2-byte formats: the sphere's drag is summed by its own kernel from the
// buffer a step reads (launch it with that step's arguments after the step)
// instead of inside the step kernel.
bool drag_in_own_kernel(Store s);
cudaError_t launch_drag_links(Store st, const StepArgs& a, cudaStream_t s);
// Deterministic FP64 sums over n values: out[c] = sum of comp(c) over cells
// for the requested quantity; partial sums of `blocks` blocks go to scratch.
enum class RedKind : int { Mass = 0, Kinetic = 1, DiffSq = 2, NormSq = 3, UMax = 4 };
int reduce_blocks();
// out[0] = sum |u - u2|^2, out[1] = sum |u|^2 in one pass (scratch: 2 values
// per reduction block, 2 * reduce_blocks()).
cudaError_t launch_residual_sums(const double* u, const double* v, const double* w, const double* u2,
                                 const double* v2, const double* w2, int64_t n, double* scratch, double* out,
                                 cudaStream_t s);
// out = sqrt(nd[0] / nd[1]) with the residual's conventions (one thread).
cudaError_t launch_residual_finish(const double* nd, int first, double* out, cudaStream_t s);
cudaError_t launch_reduce(RedKind k, const double* u, const double* v, const double* w, const double* p,
                          const double* u2, const double* v2, const double* w2, int64_t n, double* scratch,
                          double* out, cudaStream_t s);

}  // namespace imx
