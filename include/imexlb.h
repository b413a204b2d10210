/* imexlb-b200: C ABI of the B200 (sm_100a) D3Q27 lattice-Boltzmann step.
 *
 * This is the drop-in boundary for the imexlb proxy apps' solver.  The
 * reference has no library interface: its "API" is the System class (input.in
 * parsing, tgv/src/System.hpp) and the LBM struct's member functions
 * (tgv/src/lbm.hpp:238-251) called by each case's main().  Every entry point
 * below names the reference function it replaces.
 *
 * Conventions: every function returns 0 on success and a nonzero IMEXLB_E_*
 * code on failure (no exception crosses the ABI); imexlb_last_error() gives
 * the message of the calling thread's last failure.  The library owns all
 * device memory; callers own host buffers.  A lattice handle belongs to one
 * host thread at a time.  Host arrays are interior fields with x fastest:
 * index i + nx*(j + ny*k), the Fortran order MPIoutput writes
 * (tgv/src/lbm.cpp:361-377).
 */
#ifndef IMEXLB_H
#define IMEXLB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define IMEXLB_Q 27

enum {
  IMEXLB_OK = 0,
  IMEXLB_E_ARG = 1,      /* invalid argument */
  IMEXLB_E_CUDA = 2,     /* CUDA runtime error (message has the CUDA text) */
  IMEXLB_E_IO = 3,       /* file error */
  IMEXLB_E_NOMEM = 4,    /* device or host allocation failed */
  IMEXLB_E_STATE = 5,    /* call out of order, or the lattice went non-finite */
  IMEXLB_E_UNSUPPORTED = 6
};

/* The three proxy apps (tgv/, lid_driven_cavity/, sphere/). */
typedef enum imexlb_case { IMEXLB_TGV = 0, IMEXLB_CAVITY = 1, IMEXLB_SPHERE = 2 } imexlb_case;

/* Boundary treatment.
 * IMEXLB_BC_REFERENCE: the reference's own boundary passes, bit for bit,
 *   including their ghost-slot chains (lid_driven_cavity/src/lbm.cpp:231-317,
 *   sphere/src/lbm.cpp:274-371) and forced moments (Update).  TGV is
 *   periodic either way.
 * IMEXLB_BC_STANDARD: halfway bounce-back with the moving-wall correction
 *   -2 w_i rho (c_i . u_w)/cs^2 on the cavity lid; for the sphere a periodic
 *   channel with an equilibrium inlet, a zero-gradient outlet and halfway
 *   bounce-back on a voxelised sphere (momentum-exchange drag available).
 * IMEXLB_BC_SLAB (cavity only, FP64 or FP32 storage): the standard cavity's
 *   bottom wall and moving lid with x and y periodic, a lid-driven slab whose
 *   steady state is plane Couette flow u(z) = u_w (z + 1/2) / nz; it checks
 *   the moving-wall rule against that exact solution.  No counterpart in the
 *   reference.
 * IMEXLB_BC_REFERENCE_LINKS (cavity only, FP64 or FP32 storage): the same
 *   results as IMEXLB_BC_REFERENCE, bit for bit, with the boundary passes
 *   resolved per link inside the step kernel (a face-code table per face
 *   cell) instead of a gather of the ghost slots after each step. */
typedef enum imexlb_bc {
  IMEXLB_BC_REFERENCE = 0,
  IMEXLB_BC_STANDARD = 1,
  IMEXLB_BC_SLAB = 2,
  IMEXLB_BC_REFERENCE_LINKS = 3
} imexlb_bc;

/* Storage of the distributions in HBM.  F64 stores f_i; F32/F16/BF16 store
 * the deviation f_i - w_i * 3 p_ref scaled per population, and collide in FP32. */
typedef enum imexlb_storage {
  IMEXLB_F64 = 0,
  IMEXLB_F32 = 1,
  IMEXLB_F16 = 2,
  IMEXLB_BF16 = 3
} imexlb_storage;

/* FP64 arithmetic mode.  EXACT keeps the reference's operation order with
 * one rounding per operation (bit-identical to the reference); FAST lets
 * multiply-adds fuse and divides by constants become multiplies (agrees with
 * the reference to ~1e-15 relative). */
typedef enum imexlb_arith { IMEXLB_ARITH_EXACT = 0, IMEXLB_ARITH_FAST = 1 } imexlb_arith;

/* System (tgv/src/System.hpp:9-15): the nine input.in numbers and what the
 * constructor derives from them. */
typedef struct imexlb_system {
  double rho0, R;
  int Re;
  double u0;
  int Time, inter;
  int sx, sy, sz;
  double miu, tau, Ma, cs2, cs;
} imexlb_system;

typedef struct imexlb_params {
  imexlb_case kase;
  imexlb_bc bc;
  imexlb_storage storage;
  imexlb_arith arith;   /* FP64 storage only */
  int nx, ny, nz;       /* interior lattice (glx, gly, glz) */
  double tau0;          /* 3 nu: System::tau; the relaxation time is tau0 + 0.5 */
  double rho0, u0;      /* LBM::rho0, LBM::u0 */
  /* Sphere, reference boundaries: padded (nx+6)(ny+6)(nz+6) integer field
   * `ran` (x fastest) of sphere/src/lbm.cpp:221-229; NULL = derive it from
   * `seed` with this library's generator. */
  const int32_t* ran;
  uint64_t seed;
  /* Standard boundaries: lid velocity (cavity, along +x), inlet velocity,
   * sphere diameter and centre (sphere channel).  Zero = BASELINE defaults. */
  double lid_u;
  double inlet_u;
  double sphere_d;
  double sphere_c[3];
  void* stream; /* cudaStream_t to run on (it must stay valid until imexlb_destroy
                  returns); NULL = the legacy default stream */
} imexlb_params;

typedef struct imexlb_lattice imexlb_lattice;

/* Fill *p with defaults (FP64, EXACT, reference boundaries). */
void imexlb_params_default(imexlb_params* p);

/* System::System (tgv/src/System.cpp:5-24, lid_driven_cavity/src/System.cpp:5-20,
 * sphere/src/System.cpp:5-23): parse `path` (an input.in) for `kase`,
 * including the per-case overrides of Time and inter. */
int imexlb_system_read(const char* path, imexlb_case kase, imexlb_system* out);

/* LBM::LBM + LBM::Initialize (tgv/src/lbm.hpp:161-236, tgv/src/lbm.cpp:7-221):
 * allocate the lattice on the current CUDA device and set the initial state. */
int imexlb_create(const imexlb_params* p, imexlb_lattice** out);

/* LBM::Initialize again (tgv/main.cpp:68): reset to the initial state. */
int imexlb_initialize(imexlb_lattice* h);

/* nsteps x { Collision; pack; exchange; unpack; Streaming; Update }
 * (tgv/main.cpp:70-134, lid_driven_cavity/main.cpp:67-83), fused into one
 * kernel per step (plus one small ghost-slot kernel for reference
 * boundaries).  Asynchronous on the lattice's stream. */
int imexlb_step(imexlb_lattice* h, int nsteps);

/* The ua, va, wa, p views after the last step (interior, x fastest; any
 * pointer may be NULL).  Synchronises the lattice's stream. */
int imexlb_get_fields(imexlb_lattice* h, double* u, double* v, double* w, double* p);

/* The same views, asynchronously: enqueues their copy into the host
 * buffers (pinned memory lets it overlap the following steps) and returns.
 * The buffers hold the fields, and must stay allocated, until the next
 * synchronising call (imexlb_synchronize, imexlb_get_fields, ...).  The
 * next imexlb_step call's last step, which rewrites the views, waits for
 * the copy; the steps before it run meanwhile. */
int imexlb_get_fields_async(imexlb_lattice* h, double* u, double* v, double* w, double* p);

/* The usr view (sphere solid mask, 1 = fluid; interior, x fastest). */
int imexlb_get_mask(imexlb_lattice* h, int32_t* usr);

/* LBM::MPIoutput(n) at one rank (tgv/src/lbm.cpp:335-669): the 332-byte
 * #!TDV112 header and x, y, z, u, v, w, p as FP64, written to `path`. */
int imexlb_write_tecplot(imexlb_lattice* h, const char* path, int n);

/* FP64 reductions over the interior after the last step. */
enum {
  IMEXLB_REDUCE_MASS = 0,     /* sum of 3p                          */
  IMEXLB_REDUCE_KINETIC = 1,  /* sum of (u^2+v^2+w^2)/2              */
  IMEXLB_REDUCE_RESIDUAL = 2, /* sqrt(sum|u-u_prev|^2 / sum|u|^2) between the
                                 last two calls of this reduction     */
  IMEXLB_REDUCE_DRAG = 3,     /* momentum-exchange force on the sphere at the
                                 last step, out[0..2] (standard sphere) */
  IMEXLB_REDUCE_UMAX = 4      /* max |u|                             */
};
int imexlb_reduce(imexlb_lattice* h, int kind, double* out);

/* The MASS, KINETIC, UMAX or RESIDUAL reduction (one value) without waiting
 * for the GPU: the reduction and the copy of its value into `out` are queued
 * on the lattice's stream, and *out holds the value once the next
 * synchronising call (imexlb_synchronize, imexlb_get_fields, ...) returns.
 * `out` should be pinned host memory (with pageable memory the copy waits for
 * the stream).  A non-finite lattice gives NaN or an infinite value instead
 * of the IMEXLB_E_STATE that imexlb_reduce returns.  A solve loop can so check
 * its residual every few steps without stalling the steps behind it. */
int imexlb_reduce_async(imexlb_lattice* h, int kind, double* out);

/* The MASS, KINETIC and UMAX reductions over caller-provided device fields
 * (u, v, w, p, n values each; a field the reduction does not read may be
 * NULL), writing the result to the device address `out`, asynchronously on
 * `stream` (a cudaStream_t, NULL = legacy default stream).  No counterpart in
 * the reference.  It allocates nothing: for callers that may not allocate
 * device memory (an application that reserves all device memory up front, a
 * plugin inside a framework that owns every allocation, code that must avoid
 * cudaMalloc's implicit synchronisation), its partial sums live in a fixed
 * 32 KiB array inside the library that every GPU using the library holds
 * until exit.  n is limited to 268435456 cells; larger n is rejected with
 * IMEXLB_E_ARG.  The first call on a device looks up that array's device
 * address and must come before any stream capture on that device; after a
 * reset of the device's context (cudaDeviceReset) the next call finds the
 * new context and looks the address up again, so it too must come before
 * any capture.  All calls on a device share the array: calls that overlap on
 * the GPU (other streams, other threads) race and must be serialised by the
 * caller.  Nothing in the array needs to start at zero: each call overwrites
 * every partial it reads.  The result is computed on the GPU after the call
 * returns, so a non-finite field cannot be reported as an error code (as
 * imexlb_reduce reports IMEXLB_E_STATE): it shows in *out instead, which is
 * NaN when any value read is NaN (UMAX included) and infinite when one is
 * infinite. */
int imexlb_reduce_fields_noalloc(int kind, const double* u, const double* v, const double* w, const double* p,
                                 int64_t n, double* out, void* stream);

/* Number of steps taken since the last (re)initialisation. */
int imexlb_steps_taken(const imexlb_lattice* h, int64_t* steps);

/* Device bytes the lattice holds, and HBM bytes one step moves by design. */
int imexlb_footprint(const imexlb_lattice* h, size_t* device_bytes, double* bytes_per_cell_update);

/* Checkpoint / restore of a lattice's state: both distribution buffers, the
 * moments of the last step and the step count, in a host buffer of
 * imexlb_checkpoint_size bytes (a small header names the case, storage,
 * boundaries and extents).  Restoring into a lattice created with the same
 * parameters continues bit for bit as if it had never stopped; the residual
 * history starts over.  No counterpart in the reference, which has no
 * restart files; used to pre-empt and resume served solves. */
int imexlb_checkpoint_size(const imexlb_lattice* h, size_t* bytes);
int imexlb_checkpoint_save(imexlb_lattice* h, void* host, size_t bytes);
int imexlb_checkpoint_load(imexlb_lattice* h, const void* host, size_t bytes);

/* Host-only: the ghost-slot plan that reference boundaries apply after every
 * step (the reference's unpack + boundary passes at one rank, resolved into
 * one copy per slot; lid_driven_cavity/src/lbm.cpp:231-301,
 * sphere/src/lbm.cpp:274-356).  Slots are keyed as the reference stores f:
 * key = q + 27*(i + lx*(j + ly*k)) over the padded box, lx = nx + 6.  After a
 * step, slot tgt[n] takes: src[n] >= 0 -> that slot of this step's
 * post-collision state; src[n] == -1 -> zero; src[n] <= -2 -> slot
 * (-src[n] - 2) as it stood after the previous step.  usr_padded is the
 * sphere's padded solid mask (NULL for the cavity).  Call with tgt = src =
 * NULL to get the count in *n. */
int imexlb_ghost_plan(imexlb_case kase, int nx, int ny, int nz, const int32_t* usr_padded, int64_t* tgt,
                      int64_t* src, int64_t* n);

/* Per-launch device timing (CUDA events on the lattice's stream around each
 * kernel launch), for roofline measurement.  imexlb_profile(h, 1) starts
 * recording, imexlb_profile_read() waits, sums the durations since the start
 * and stops recording.  No counterpart in the reference (it times phases
 * with MPI_Wtime, tgv/main.cpp:74-119). */
typedef struct imexlb_kernel_times {
  double step_ms;  /* fused step kernels */
  double ghost_ms; /* ghost-slot gathers (reference boundaries) */
  int64_t step_launches, ghost_launches;
} imexlb_kernel_times;
int imexlb_profile(imexlb_lattice* h, int enable);
int imexlb_profile_read(imexlb_lattice* h, imexlb_kernel_times* out);

/* Wait for all work queued on the lattice's stream. */
int imexlb_synchronize(imexlb_lattice* h);

/* Bound, in (0, 1] seconds (default 1), on each wait of the 2-byte staged
 * step kernels for their own row copies or for a stage to be released.  A
 * block that waits longer gives up: it lets its copies in flight land (that
 * drain keeps the full second), leaves, and the next synchronising call
 * returns IMEXLB_E_CUDA ("gave up waiting"); a bound below a microsecond
 * gives up after one failed poll.  The lattice state is then
 * invalid until imexlb_initialize or a checkpoint load.  Lets a caller, or a
 * test, exercise that failure path without a fault.  No counterpart in the
 * reference. */
int imexlb_set_wait_limit(imexlb_lattice* h, double seconds);

/* Rounding of the FP16 / BF16 stores: 1 = stochastic (the default for the
 * cavity and the sphere channel: a pseudo-random fraction of a unit in the
 * last place, from a hash of cell, population and step count, is added
 * before rounding toward zero, so the rounding error is zero on average and
 * does not accumulate in a steady flow), 0 = to nearest (the vortex's only
 * mode).  IMEXLB_E_UNSUPPORTED for stochastic rounding of another storage
 * format or of the vortex.  No counterpart in the reference. */
int imexlb_set_rounding(imexlb_lattice* h, int stochastic);

void imexlb_destroy(imexlb_lattice* h);

/* Lattices take their device memory from a stream-ordered pool per device
 * that keeps up to 16 GiB of freed memory reserved, so that a lattice created
 * after another was destroyed maps no new memory and does not wait for the
 * device.  This returns the reserved memory of the current device to the
 * system (it waits for the device first).  No counterpart in the reference. */
int imexlb_release_cached_memory(void);

/* Message of the calling thread's last failure ("" if none). */
const char* imexlb_last_error(void);

/* ------------------------------------------------------------ engine
 * Many independent lattices ("instances") on one GPU, every active one
 * advanced one time step per persistent kernel launch over a device-side
 * (instance, tile) work list; the steps run as CUDA-graph replays while the
 * set of instances is unchanged.  Instances live in one device arena
 * reserved at creation (budget_bytes); an instance that does not fit is
 * refused with IMEXLB_E_NOMEM, so a server admits work against an HBM
 * budget.  Instances can be added and removed between any two steps.
 * Supported instance kinds: TGV (periodic), lid-driven cavity and sphere
 * channel with standard boundaries (IMEXLB_BC_STANDARD semantics), in the
 * engine's storage format.  No counterpart in the reference, which runs one
 * lattice per process (BASELINE batched and served configurations). */
typedef struct imexlb_engine imexlb_engine;

typedef struct imexlb_instance_desc {
  imexlb_case kase;
  int nx, ny, nz;
  double tau0, rho0, u0;  /* as imexlb_params */
  double lid_u, inlet_u, sphere_d, sphere_c[3];  /* 0 = defaults (u0, u0, nx/24, (nx/4, ny/2, nz/2)) */
  int tile_bx; /* threads along x per tile (power of two, 8..256); 0 = default (2-byte formats: whole rows
                  staged in shared memory where a row fits) */
} imexlb_instance_desc;

typedef struct imexlb_engine_stats {
  int instances;
  int64_t cells;
  size_t budget_bytes, used_bytes;
  int64_t tiles, steps;
} imexlb_engine_stats;

int imexlb_engine_create(imexlb_storage storage, imexlb_arith arith, size_t budget_bytes, int max_instances,
                         void* stream, imexlb_engine** out);
/* Add an instance (initial state as imexlb_create); *slot identifies it.
 * Returns without waiting for the GPU: the instance's uploads and set-up
 * follow the work already queued on the engine's stream, so a host can admit
 * while earlier steps run. */
int imexlb_engine_add(imexlb_engine* e, const imexlb_instance_desc* d, int* slot);
/* The same in a storage format of its own: one engine holds instances of
 * several formats (each format's instances run their own kernel groups in
 * the same step launches and graph), so a caller can store in FP16 the
 * instances whose relaxation is far enough from 1/2 and in FP32 the
 * marginally stable ones.  imexlb_engine_create's storage is the format of
 * imexlb_engine_add. */
int imexlb_engine_add_as(imexlb_engine* e, const imexlb_instance_desc* d, imexlb_storage storage, int* slot);
int imexlb_engine_remove(imexlb_engine* e, int slot);
/* Every active instance advances nsteps steps; the moments of the last are stored. */
int imexlb_engine_step(imexlb_engine* e, int nsteps);
/* Step limit of one instance: it takes at most `steps` more steps (< 0: no
 * limit, the default at admission), then stays as it is while the others go
 * on; its u, v, w, p views are written at its last step.  A serving loop can
 * so run fixed-length step calls over requests of any step count.  The new
 * limit applies from the next imexlb_engine_step call on (steps already
 * queued keep the old one); the call does not wait for the GPU. */
int imexlb_engine_limit(imexlb_engine* e, int slot, int steps);
/* u, v, w, p of one instance after the last step (host arrays, x fastest). */
int imexlb_engine_fields(imexlb_engine* e, int slot, double* u, double* v, double* w, double* p);
/* The same for one z plane k of the instance (nx * ny values each, x
 * fastest): a compact answer for a serving loop whose requests want a cut
 * through the flow rather than the whole field. */
int imexlb_engine_plane(imexlb_engine* e, int slot, int k, double* u, double* v, double* w, double* p);
/* Velocity residual per slot, sqrt(sum|u - u_prev|^2 / sum|u|^2) between this
 * call and the previous one (INFINITY on an instance's first call, -1 for an
 * instance that took no step since the previous call -- it stopped at its
 * step limit, which is not convergence --, NaN for empty slots or a
 * non-finite lattice); out has max_instances entries.  Call it right after
 * imexlb_engine_step. */
int imexlb_engine_residuals(imexlb_engine* e, double* out, int n_out);
int imexlb_engine_info(const imexlb_engine* e, imexlb_engine_stats* st);
/* Arena bytes one instance needs in a given storage format. */
int imexlb_engine_instance_bytes(imexlb_storage storage, const imexlb_instance_desc* d, size_t* bytes);
/* Pre-emption of one engine instance: its state (current distribution
 * buffer, moments, step count) into a host buffer, and admission of an
 * instance from such a buffer (same descriptor; the instance keeps the
 * checkpoint's storage format), which then continues bit for bit.  The restored instance's residual history starts
 * over.  No counterpart in the reference. */
int imexlb_engine_checkpoint_size(const imexlb_engine* e, int slot, size_t* bytes);
int imexlb_engine_checkpoint_save(imexlb_engine* e, int slot, void* host, size_t bytes);
int imexlb_engine_restore(imexlb_engine* e, const imexlb_instance_desc* d, const void* host, size_t bytes,
                          int* slot);
int imexlb_engine_synchronize(imexlb_engine* e);
void imexlb_engine_destroy(imexlb_engine* e);

/* Library version string. */
const char* imexlb_version(void);

#ifdef __cplusplus
}
#endif
#endif /* IMEXLB_H */
