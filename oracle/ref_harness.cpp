// Test infrastructure: drives the reference proxy app's own solver (its
// System, LBM::Initialize/Collision/pack/exchange/unpack/Streaming/Update and
// MPIoutput, compiled from the reference sources against oracle/refshim) and
// exports its state through a C ABI for the pinning tests and the CPU
// baseline.  Built once per case (REF_CASE_TGV / REF_CASE_CAVITY /
// REF_CASE_SPHERE) by oracle/Makefile into oracle/_ref/.
//
// Call sequence restated from the drivers:
//   tgv/main.cpp:37-134               ctor, Initialize, setup_subdomain,
//                                     20 warm-up steps, Initialize, timed loop
//   lid_driven_cavity/main.cpp:60-83  ctor, Initialize, MPIoutput(0),
//                                     setup_subdomain, loop with MPIoutput
//                                     every `inter` steps
//   sphere/main.cpp                   ctor, Initialize, setup_subdomain, loop
// Two undefined reads of the reference are pinned here, as documented:
//   * LBM::cs2 is never assigned (tgv/src/lbm.hpp:135) but read by the TGV
//     initial pressure (tgv/src/lbm.cpp:202): pinned to 1/3, System's value.
//   * the cavity's never-received halo buffers (malloc'd in
//     lid_driven_cavity/src/mpi_view_transfer.cpp:3-82) are copied into four
//     ghost planes by unpack at one rank: pinned to zero.
#include <unistd.h>

#include <cstring>
#include <string>

#include "System.hpp"

namespace {

struct Cwd {
  std::string old;
  bool ok = false;
  explicit Cwd(const char* dir) {
    char buf[4096];
    if (getcwd(buf, sizeof buf)) old = buf;
    ok = dir && chdir(dir) == 0;
  }
  ~Cwd() {
    if (!old.empty()) (void)chdir(old.c_str());
  }
};

#if defined(REF_CASE_TGV)
System make_system() { return System(0); }
#else
System make_system() { return System(); }
#endif

void zero_halo_buffers(LBM& l) {
#if defined(REF_CASE_CAVITY)
  const size_t face_y = sizeof(double) * q * l.lx * l.lz;
  const size_t face_z = sizeof(double) * q * l.lx * l.ly;
  const size_t face_x = sizeof(double) * q * l.ly * l.lz;
  std::memset(l.m_front, 0, face_y);
  std::memset(l.m_frontout, 0, face_y);
  std::memset(l.m_back, 0, face_y);
  std::memset(l.m_backout, 0, face_y);
  std::memset(l.m_up, 0, face_z);
  std::memset(l.m_upout, 0, face_z);
  std::memset(l.m_down, 0, face_z);
  std::memset(l.m_downout, 0, face_z);
  std::memset(l.m_left, 0, face_x);
  std::memset(l.m_leftout, 0, face_x);
  std::memset(l.m_right, 0, face_x);
  std::memset(l.m_rightout, 0, face_x);
#else
  (void)l;
#endif
}

void export_state(LBM& l, double* u, double* v, double* w, double* p, int* usr, int* ran, double* f) {
  const int nx = l.l_l[0], ny = l.l_l[1], nz = l.l_l[2];
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const size_t o = i + static_cast<size_t>(nx) * (j + static_cast<size_t>(ny) * k);
        if (u) u[o] = l.ua(i + ghost, j + ghost, k + ghost);
        if (v) v[o] = l.va(i + ghost, j + ghost, k + ghost);
        if (w) w[o] = l.wa(i + ghost, j + ghost, k + ghost);
        if (p) p[o] = l.p(i + ghost, j + ghost, k + ghost);
      }
  const size_t cells = static_cast<size_t>(l.lx) * l.ly * l.lz;
  if (usr) std::memcpy(usr, l.usr.data(), cells * sizeof(int));
  if (ran) std::memcpy(ran, l.ran.data(), cells * sizeof(int));
  if (f) std::memcpy(f, l.f.data(), cells * q * sizeof(double));
}

void step(LBM& l) {
  l.Collision();
  l.pack();
  l.exchange();
  l.unpack();
  l.Streaming();
  l.Update();
}

}  // namespace

extern "C" {

struct ref_system {
  double rho0, R;
  int Re;
  double u0;
  int Time, inter;
  int sx, sy, sz;
  double miu, tau, Ma, cs2, cs;
};

// System::System on `dir`/input.in.
int ref_read_system(const char* dir, ref_system* out) {
  Cwd cwd(dir);
  if (!cwd.ok) return 1;
  System s = make_system();
  out->rho0 = s.rho0;
  out->R = s.R;
  out->Re = s.Re;
  out->u0 = s.u0;
  out->Time = s.Time;
  out->inter = s.inter;
  out->sx = s.sx;
  out->sy = s.sy;
  out->sz = s.sz;
  out->miu = s.miu;
  out->tau = s.tau;
  out->Ma = s.Ma;
  out->cs2 = s.cs2;
  out->cs = s.cs;
  return 0;
}

// Run the reference for `nsteps` steps from `dir`/input.in (the step count of
// input.in and System's overrides are ignored; `warmup` only applies to TGV,
// whose driver re-initialises after it).  With out_every > 0 MPIoutput writes
// output<n>.plt into `dir` at step 0 (cavity) and every out_every steps.
// Outputs: interior u,v,w,p (x fastest), padded usr and ran (lx*ly*lz, x
// fastest) and the padded distributions f (q*lx*ly*lz, population fastest).
// Any output pointer may be null.
int ref_run(const char* dir, int nsteps, int warmup, int out_every, double* u, double* v, double* w, double* p,
            int* usr, int* ran, double* f) {
  Cwd cwd(dir);
  if (!cwd.ok) return 1;
  System s = make_system();
  LBM l(MPI_COMM_WORLD, s.sx, s.sy, s.sz, s.tau, s.rho0, s.u0);
  l.cs2 = 1.0 / 3.0;
  l.Initialize();
#if defined(REF_CASE_CAVITY)
  if (out_every > 0) l.MPIoutput(0);
#endif
  l.setup_subdomain();
  zero_halo_buffers(l);
#if defined(REF_CASE_TGV)
  for (int it = 1; it <= warmup; ++it) step(l);
  l.Initialize();
#else
  (void)warmup;
#endif
  for (int it = 1; it <= nsteps; ++it) {
    step(l);
#if !defined(REF_CASE_SPHERE)
    if (out_every > 0 && it % out_every == 0) l.MPIoutput(it / out_every);
#endif
  }
  export_state(l, u, v, w, p, usr, ran, f);
  return 0;
}

// Padded extents (lx, ly, lz) the reference allocates for `dir`/input.in.
int ref_extents(const char* dir, int* lx, int* ly, int* lz) {
  Cwd cwd(dir);
  if (!cwd.ok) return 1;
  System s = make_system();
  *lx = s.sx + 2 * ghost;
  *ly = s.sy + 2 * ghost;
  *lz = s.sz + 2 * ghost;
  return 0;
}

}  // extern "C"
