/* CPU restatement of the imexlb D3Q27 step -- TEST INFRASTRUCTURE ONLY.
 *
 * It is the checker for the parity tests, smoke() and the cpu_baseline leg of
 * bench.py, never part of the product path.  Every function below restates a
 * reference function (file:line given with each) in the same loop structure,
 * with the same expression order, so that built with -ffp-contract=off it
 * reproduces the reference's arithmetic bit for bit; tests/test_oracle_pinning.py
 * checks exactly that against the reference's own sources built in oracle/_ref.
 *
 * The only deliberate departure from a literal transcription: pow(x, 2)
 * appears as x * x.  g++ folds the reference's pow(double, 2) into x * x, and
 * for the integer arguments of the sphere mask the square is exact either way.
 */
#include "imexlb_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define Q 27
#define GHOST 3
#define PI_REF 3.1415926 /* tgv/src/lbm.cpp:5 */

struct oracle_lbm {
  int kase;
  int nx, ny, nz; /* glx, gly, glz (one rank: l_l == gl) */
  int lx, ly, lz; /* padded */
  int ls[3], le[3];
  double tau0, rho0, u0, cs2;
  double* f;
  double* ft;
  double *ua, *va, *wa, *p;
  int* usr;
  int* ran;
  double t[Q];
  int bb[Q];
  int e[Q][3];
};

/* tgv/src/lbm.cpp:27-190 (identical in the three cases) */
static const double W_REF[Q] = {8.0 / 27.0, 2.0 / 27.0,  2.0 / 27.0,  2.0 / 27.0,  2.0 / 27.0,  2.0 / 27.0,
                                2.0 / 27.0, 1.0 / 54.0,  1.0 / 54.0,  1.0 / 54.0,  1.0 / 54.0,  1.0 / 54.0,
                                1.0 / 54.0, 1.0 / 54.0,  1.0 / 54.0,  1.0 / 54.0,  1.0 / 54.0,  1.0 / 54.0,
                                1.0 / 54.0, 1.0 / 216.0, 1.0 / 216.0, 1.0 / 216.0, 1.0 / 216.0, 1.0 / 216.0,
                                1.0 / 216.0, 1.0 / 216.0, 1.0 / 216.0};
static const int BB_REF[Q] = {0,  2,  1,  4,  3,  6,  5,  8,  7,  10, 9,  12, 11, 14,
                              13, 16, 15, 18, 17, 20, 19, 22, 21, 24, 23, 26, 25};
static const int E_REF[Q][3] = {{0, 0, 0},   {1, 0, 0},   {-1, 0, 0},  {0, 1, 0},   {0, -1, 0},   {0, 0, 1},
                                {0, 0, -1},  {1, 1, 0},   {-1, -1, 0}, {1, -1, 0},  {-1, 1, 0},   {1, 0, 1},
                                {-1, 0, -1}, {1, 0, -1},  {-1, 0, 1},  {0, 1, 1},   {0, -1, -1},  {0, 1, -1},
                                {0, -1, 1},  {1, 1, 1},   {-1, -1, -1}, {1, -1, 1}, {-1, 1, -1},  {1, 1, -1},
                                {-1, -1, 1}, {1, -1, -1}, {-1, 1, 1}};

static inline size_t C3(const oracle_lbm* o, int i, int j, int k) {
  return (size_t)i + (size_t)o->lx * ((size_t)j + (size_t)o->ly * (size_t)k);
}
static inline size_t F4(const oracle_lbm* o, int ii, int i, int j, int k) {
  return (size_t)ii + Q * C3(o, i, j, k);
}
#define FV(o, ii, i, j, k) ((o)->f[F4((o), (ii), (i), (j), (k))])

int oracle_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

oracle_lbm* oracle_create(int kase, int nx, int ny, int nz, double tau0, double rho0, double u0,
                          const int* ran_padded) {
  if (kase < 0 || kase > 2 || nx < 2 || ny < 2 || nz < 2) return NULL;
  oracle_lbm* o = (oracle_lbm*)calloc(1, sizeof(oracle_lbm));
  if (!o) return NULL;
  o->kase = kase;
  o->nx = nx;
  o->ny = ny;
  o->nz = nz;
  o->lx = nx + 2 * GHOST; /* tgv/src/lbm.hpp:168-178 */
  o->ly = ny + 2 * GHOST;
  o->lz = nz + 2 * GHOST;
  o->ls[0] = o->ls[1] = o->ls[2] = GHOST;
  o->le[0] = GHOST + nx;
  o->le[1] = GHOST + ny;
  o->le[2] = GHOST + nz;
  o->tau0 = tau0;
  o->rho0 = rho0;
  o->u0 = u0;
  o->cs2 = 1.0 / 3.0; /* LBM::cs2 is read uninitialised by the TGV init; pinned to System's 1/3 */
  const size_t cells = (size_t)o->lx * o->ly * o->lz;
  o->f = (double*)calloc(cells * Q, sizeof(double));
  o->ft = (double*)calloc(cells * Q, sizeof(double));
  o->ua = (double*)calloc(cells, sizeof(double));
  o->va = (double*)calloc(cells, sizeof(double));
  o->wa = (double*)calloc(cells, sizeof(double));
  o->p = (double*)calloc(cells, sizeof(double));
  o->usr = (int*)calloc(cells, sizeof(int));
  o->ran = (int*)calloc(cells, sizeof(int));
  if (!o->f || !o->ft || !o->ua || !o->va || !o->wa || !o->p || !o->usr || !o->ran) {
    oracle_destroy(o);
    return NULL;
  }
  if (ran_padded) memcpy(o->ran, ran_padded, cells * sizeof(int));
  for (int ii = 0; ii < Q; ++ii) {
    o->t[ii] = W_REF[ii];
    o->bb[ii] = BB_REF[ii];
    for (int d = 0; d < 3; ++d) o->e[ii][d] = E_REF[ii][d];
  }
  return o;
}

void oracle_destroy(oracle_lbm* o) {
  if (!o) return;
  free(o->f);
  free(o->ft);
  free(o->ua);
  free(o->va);
  free(o->wa);
  free(o->p);
  free(o->usr);
  free(o->ran);
  free(o);
}

/* feq of tgv/src/lbm.cpp:211-215 (initf) and :228-232 (collision), with the
 * reference's tables t = W_REF, e = E_REF and its expression order.  The
 * standard-boundary variants below use this function too. */
static inline double feq_tab(int ii, double u, double v, double w, double p) {
  const double e0 = E_REF[ii][0], e1 = E_REF[ii][1], e2 = E_REF[ii][2];
  const double t = W_REF[ii];
  const double edu = e0 * u + e1 * v + e2 * w;
  const double udu = u * u + v * v + w * w;
  const double eu2 = (e0 * u + e1 * v + e2 * w) * (e0 * u + e1 * v + e2 * w);
  return t * p * 3.0 + t * (3.0 * edu + 4.5 * eu2 - 1.5 * udu);
}

static inline double feq_ref(const oracle_lbm* o, int ii, double u, double v, double w, double p) {
  (void)o; /* o->t and o->e are copies of W_REF and E_REF */
  return feq_tab(ii, u, v, w, p);
}

/* One population's collision, tgv/src/lbm.cpp:233: f -= (f - feq)/(tau0 + 0.5) */
static inline double collide_ref(double f, double feq, double tau0) { return f - (f - feq) / (tau0 + 0.5); }

/* Moments of one cell's populations as the cavity and sphere Update sum them
 * (lid_driven_cavity/src/lbm.cpp:330-339, sphere/src/lbm.cpp:385-394): one
 * loop over the populations in order from zero accumulators. */
static inline void moments_ref(const double* fc, double* p, double* u, double* v, double* w) {
  double pm = 0.0, um = 0.0, vm = 0.0, wm = 0.0;
  for (int ii = 0; ii < Q; ++ii) {
    pm = pm + fc[ii] / 3.0;
    um = um + fc[ii] * E_REF[ii][0];
    vm = vm + fc[ii] * E_REF[ii][1];
    wm = wm + fc[ii] * E_REF[ii][2];
  }
  *p = pm;
  *u = um;
  *v = vm;
  *w = wm;
}

/* ------------------------------------------------------------ Initialize */
static void init_tgv(oracle_lbm* o) { /* tgv/src/lbm.cpp:195-206 */
  const int glx = o->nx, gly = o->ny, glz = o->nz;
  const double u0 = o->u0, rho0 = o->rho0, cs2 = o->cs2;
#pragma omp parallel for schedule(static)
  for (int k = 0; k < o->lz; ++k)
    for (int j = 0; j < o->ly; ++j)
      for (int i = 0; i < o->lx; ++i) {
        const double X = (double)(i - GHOST + 0) / (double)glx * 2.0 * PI_REF;
        const double Y = (double)(j - GHOST + 0) / (double)gly * 2.0 * PI_REF;
        const double Z = (double)(k - GHOST + 0) / (double)glz * 2.0 * PI_REF;
        const size_t c = C3(o, i, j, k);
        o->ua[c] = u0 * sin(X) * cos(Y) * cos(Z);
        o->va[c] = -u0 * cos(X) * sin(Y) * cos(Z);
        o->wa[c] = 0;
        o->p[c] = rho0 * cs2 + rho0 * u0 * u0 / 16.0 * (cos(X * 2.0) + cos(Y * 2.0)) * (cos(Z * 2.0) + 2.0);
      }
}

static void init_cavity(oracle_lbm* o) { /* lid_driven_cavity/src/lbm.cpp:191-198 */
  const size_t cells = (size_t)o->lx * o->ly * o->lz;
  memset(o->ua, 0, cells * sizeof(double));
  memset(o->va, 0, cells * sizeof(double));
  memset(o->wa, 0, cells * sizeof(double));
  memset(o->p, 0, cells * sizeof(double));
}

static void init_sphere(oracle_lbm* o) { /* sphere/src/lbm.cpp:231-242 (ran given) */
  const int glx = o->nx, glz = o->nz;
  const double u0 = o->u0;
  const int c8 = (glx - 1) / 8;
  const double r = (glx - 1) / 64.0;
#pragma omp parallel for schedule(static)
  for (int k = 0; k < o->lz; ++k)
    for (int j = 0; j < o->ly; ++j)
      for (int i = 0; i < o->lx; ++i) {
        const size_t c = C3(o, i, j, k);
        const int dx = 0 + i - GHOST - c8, dy = 0 + j - GHOST - c8, dz = 0 + k - GHOST - c8;
        const double d2 = (double)dx * (double)dx + (double)dy * (double)dy + (double)dz * (double)dz;
        o->usr[c] = (d2 <= r * r) ? 0 : 1;
        o->ua[c] = (u0 * 4.0 * (0 + k - GHOST) * (glz - 1 - (0 + k - GHOST)) / ((double)(glz - 1) * (double)(glz - 1))) *
                   o->usr[c] * (1.0 + o->ran[c] * 0.001);
        o->va[c] = 0.0;
        o->wa[c] = 0.0;
        o->p[c] = 0;
      }
}

void oracle_initialize(oracle_lbm* o) {
  const size_t cells = (size_t)o->lx * o->ly * o->lz;
  memset(o->f, 0, cells * Q * sizeof(double));
  memset(o->ft, 0, cells * Q * sizeof(double));
  if (o->kase == ORACLE_TGV) init_tgv(o);
  if (o->kase == ORACLE_CAVITY) init_cavity(o);
  if (o->kase == ORACLE_SPHERE) init_sphere(o);
  /* initf: f = feq over the whole padded box, ft = 0 (tgv/src/lbm.cpp:209-218) */
#pragma omp parallel for schedule(static)
  for (int k = 0; k < o->lz; ++k)
    for (int j = 0; j < o->ly; ++j)
      for (int i = 0; i < o->lx; ++i) {
        const size_t c = C3(o, i, j, k);
        for (int ii = 0; ii < Q; ++ii) o->f[ii + Q * c] = feq_ref(o, ii, o->ua[c], o->va[c], o->wa[c], o->p[c]);
      }
}

/* ------------------------------------------------------------ Collision */
void oracle_collision(oracle_lbm* o) { /* tgv/src/lbm.cpp:222-237 */
  const double tau0 = o->tau0;
#pragma omp parallel for schedule(static)
  for (int k = o->ls[2]; k < o->le[2]; ++k)
    for (int j = o->ls[1]; j < o->le[1]; ++j)
      for (int i = o->ls[0]; i < o->le[0]; ++i) {
        const size_t c = C3(o, i, j, k);
        for (int ii = 0; ii < Q; ++ii) {
          const double feq = feq_ref(o, ii, o->ua[c], o->va[c], o->wa[c], o->p[c]);
          double* fp = &o->f[ii + Q * c];
          *fp = collide_ref(*fp, feq, tau0);
        }
      }
}

/* ------------------------------------------------------------ halo at one rank */
static inline int wrap(int c, int n) { return c < GHOST ? c + n : (c >= GHOST + n ? c - n : c); }

void oracle_halo(oracle_lbm* o) {
  if (o->kase == ORACLE_TGV) {
    /* tgv/src/mpi_view_transfer.cpp:117-383 at one rank: every neighbour is
     * the rank itself, the 26 self-messages carry interior planes [3,6) and
     * [N,N+3) to the opposite ghost planes; the face unpacks first leave stale
     * edge/corner ghosts which the edge and corner unpacks then overwrite.
     * Net effect: every ghost cell holds the interior cell at the periodic
     * image of its coordinates. */
#pragma omp parallel for schedule(static)
    for (int k = 0; k < o->lz; ++k)
      for (int j = 0; j < o->ly; ++j)
        for (int i = 0; i < o->lx; ++i) {
          const int si = wrap(i, o->nx), sj = wrap(j, o->ny), sk = wrap(k, o->nz);
          if (si == i && sj == j && sk == k) continue;
          memcpy(&o->f[F4(o, 0, i, j, k)], &o->f[F4(o, 0, si, sj, sk)], Q * sizeof(double));
        }
  } else if (o->kase == ORACLE_CAVITY) {
    /* lid_driven_cavity/src/mpi_view_transfer.cpp:598-690 at one rank: no
     * message is sent or received, but four unpack loops are guarded by
     * `== boundary` and copy never-received malloc buffers (pinned to zero)
     * into ghost planes y = l_e1 (:617-630), z = l_e2 (:632-645),
     * x = l_s0 - 1 (:662-674) and x = l_e0 (:676-688). */
    for (int k = 0; k < o->lz; ++k)
      for (int i = 0; i < o->lx; ++i) memset(&o->f[F4(o, 0, i, o->le[1], k)], 0, Q * sizeof(double));
    for (int j = 0; j < o->ly; ++j)
      for (int i = 0; i < o->lx; ++i) memset(&o->f[F4(o, 0, i, j, o->le[2])], 0, Q * sizeof(double));
    for (int k = 0; k < o->lz; ++k)
      for (int j = 0; j < o->ly; ++j) {
        memset(&o->f[F4(o, 0, o->ls[0] - 1, j, k)], 0, Q * sizeof(double));
        memset(&o->f[F4(o, 0, o->le[0], j, k)], 0, Q * sizeof(double));
      }
  }
  /* sphere/src/mpi_view_transfer.cpp:116-439 at one rank: pack fills buffers
   * nobody reads and every unpack is guarded `!= boundary`: no effect. */
}

/* ------------------------------------------------------------ Streaming */
static void stream_interior(oracle_lbm* o) { /* tgv/src/lbm.cpp:243-253 */
#pragma omp parallel for schedule(static)
  for (int k = GHOST; k < o->lz - GHOST; ++k)
    for (int j = GHOST; j < o->ly - GHOST; ++j)
      for (int i = GHOST; i < o->lx - GHOST; ++i)
        for (int ii = 0; ii < Q; ++ii)
          o->ft[F4(o, ii, i, j, k)] = FV(o, ii, i - o->e[ii][0], j - o->e[ii][1], k - o->e[ii][2]);
#pragma omp parallel for schedule(static)
  for (int k = GHOST; k < o->lz - GHOST; ++k)
    for (int j = GHOST; j < o->ly - GHOST; ++j)
      for (int i = GHOST; i < o->lx - GHOST; ++i)
        for (int ii = 0; ii < Q; ++ii) o->f[F4(o, ii, i, j, k)] = o->ft[F4(o, ii, i, j, k)];
}

/* The wall passes read populations whose normal velocity points out of the
 * fluid and write those pointing in, so no pass reads a slot it writes; a
 * pass may run in any order internally.  Passes run in the reference order. */
static void wall_x(oracle_lbm* o, int low) { /* bcl / bcr of the cavity */
  const int e_sign = low ? 1 : -1;
  const int gx = low ? o->ls[0] - 1 : o->le[0];
  const int sx = low ? o->ls[0] + 1 : o->le[0] - 2;
#pragma omp parallel for schedule(static)
  for (int k = GHOST - 1; k < o->lz - GHOST + 1; ++k)
    for (int j = GHOST - 1; j < o->ly - GHOST + 1; ++j)
      for (int ii = 0; ii < Q; ++ii) {
        if (o->e[ii][0] * e_sign <= 0) continue;
        FV(o, ii, gx, j, k) = FV(o, o->bb[ii], sx, j + 2 * o->e[ii][1], k + 2 * o->e[ii][2]);
      }
}

static void wall_y(oracle_lbm* o, int low) { /* bcf / bcb */
  const int e_sign = low ? 1 : -1;
  const int gy = low ? o->ls[1] - 1 : o->le[1];
  const int sy = low ? o->ls[1] + 1 : o->le[1] - 2;
#pragma omp parallel for schedule(static)
  for (int k = GHOST - 1; k < o->lz - GHOST + 1; ++k)
    for (int i = GHOST - 1; i < o->lx - GHOST + 1; ++i)
      for (int ii = 0; ii < Q; ++ii) {
        if (o->e[ii][1] * e_sign <= 0) continue;
        FV(o, ii, i, gy, k) = FV(o, o->bb[ii], i + 2 * o->e[ii][0], sy, k + 2 * o->e[ii][2]);
      }
}

/* jscale = 2 normally; the cavity's top wall uses j + e(ii,1)
 * (lid_driven_cavity/src/lbm.cpp:298). */
static void wall_z(oracle_lbm* o, int low, int jscale) { /* bcd / bcu */
  const int e_sign = low ? 1 : -1;
  const int gz = low ? o->ls[2] - 1 : o->le[2];
  const int sz = low ? o->ls[2] + 1 : o->le[2] - 2;
#pragma omp parallel for schedule(static)
  for (int j = GHOST - 1; j < o->ly - GHOST + 1; ++j)
    for (int i = GHOST - 1; i < o->lx - GHOST + 1; ++i)
      for (int ii = 0; ii < Q; ++ii) {
        if (o->e[ii][2] * e_sign <= 0) continue;
        FV(o, ii, i, j, gz) = FV(o, o->bb[ii], i + 2 * o->e[ii][0], j + jscale * o->e[ii][1], sz);
      }
}

void oracle_streaming(oracle_lbm* o) {
  if (o->kase == ORACLE_CAVITY) {
    /* lid_driven_cavity/src/lbm.cpp:231-317: bcl, bcr, bcf, bcb, bcd, bcu */
    wall_x(o, 1);
    wall_x(o, 0);
    wall_y(o, 1);
    wall_y(o, 0);
    wall_z(o, 1, 2);
    wall_z(o, 0, 1);
  } else if (o->kase == ORACLE_SPHERE) {
    /* sphere/src/lbm.cpp:274-356: bcf, bcb, bcd, bcu, bcl, bcr, usrbc */
    wall_y(o, 1);
    wall_y(o, 0);
    wall_z(o, 1, 2);
    wall_z(o, 0, 2);
    /* bcl, :326-335: inlet copies the first interior plane */
#pragma omp parallel for schedule(static)
    for (int k = GHOST - 1; k < o->lz - GHOST + 1; ++k)
      for (int j = GHOST - 1; j < o->ly - GHOST + 1; ++j)
        for (int ii = 0; ii < Q; ++ii)
          if (o->e[ii][0] > 0) FV(o, ii, GHOST - 1, j, k) = FV(o, ii, GHOST, j, k);
    /* bcr, :338-347: outlet takes the upstream neighbour along -e */
    const int xe = o->le[0];
#pragma omp parallel for schedule(static)
    for (int k = GHOST - 1; k < o->lz - GHOST + 1; ++k)
      for (int j = GHOST - 1; j < o->ly - GHOST + 1; ++j)
        for (int ii = 0; ii < Q; ++ii)
          if (o->e[ii][0] < 0) FV(o, ii, xe, j, k) = FV(o, ii, xe + o->e[ii][0], j + o->e[ii][1], k + o->e[ii][2]);
    /* usrbc, :350-356: a solid cell whose neighbour along e is fluid takes
     * the reflected population two cells out.  Reads are gathered before any
     * write, the race-free reading of the parallel kernel (for a convex body
     * the sources are never written in this pass).  ft is free scratch
     * here: stream_interior overwrites it next. */
    for (int k = GHOST; k < o->lz - GHOST; ++k)
      for (int j = GHOST; j < o->ly - GHOST; ++j)
        for (int i = GHOST; i < o->lx - GHOST; ++i) {
          if (o->usr[C3(o, i, j, k)] != 0) continue;
          for (int ii = 0; ii < Q; ++ii) {
            if (o->usr[C3(o, i + o->e[ii][0], j + o->e[ii][1], k + o->e[ii][2])] != 1) continue;
            o->ft[F4(o, ii, i, j, k)] =
                FV(o, o->bb[ii], i + 2 * o->e[ii][0], j + 2 * o->e[ii][1], k + 2 * o->e[ii][2]);
          }
        }
    for (int k = GHOST; k < o->lz - GHOST; ++k)
      for (int j = GHOST; j < o->ly - GHOST; ++j)
        for (int i = GHOST; i < o->lx - GHOST; ++i) {
          if (o->usr[C3(o, i, j, k)] != 0) continue;
          for (int ii = 0; ii < Q; ++ii)
            if (o->usr[C3(o, i + o->e[ii][0], j + o->e[ii][1], k + o->e[ii][2])] == 1)
              FV(o, ii, i, j, k) = o->ft[F4(o, ii, i, j, k)];
        }
  }
  stream_interior(o);
}

/* ------------------------------------------------------------ Update */
void oracle_update(oracle_lbm* o) {
  if (o->kase == ORACLE_TGV) {
    /* tgv/src/lbm.cpp:288-333: whole padded box, sums in population order */
#pragma omp parallel for schedule(static)
    for (int k = 0; k < o->lz; ++k)
      for (int j = 0; j < o->ly; ++j)
        for (int i = 0; i < o->lx; ++i) {
          const size_t c = C3(o, i, j, k);
          const double* fc = &o->f[Q * c];
          double um = 0.0, vm = 0.0, wm = 0.0, pm = 0.0;
          for (int ii = 0; ii < Q; ++ii) um += fc[ii] * o->e[ii][0];
          for (int ii = 0; ii < Q; ++ii) vm += fc[ii] * o->e[ii][1];
          for (int ii = 0; ii < Q; ++ii) wm += fc[ii] * o->e[ii][2];
          for (int ii = 0; ii < Q; ++ii) pm += fc[ii] / 3.0;
          o->ua[c] = um;
          o->va[c] = vm;
          o->wa[c] = wm;
          o->p[c] = pm;
        }
    return;
  }
  /* lid_driven_cavity/src/lbm.cpp:319-349 and sphere/src/lbm.cpp:374-417:
   * zero all moments, then a serial interior loop */
  const size_t cells = (size_t)o->lx * o->ly * o->lz;
  memset(o->ua, 0, cells * sizeof(double));
  memset(o->va, 0, cells * sizeof(double));
  memset(o->wa, 0, cells * sizeof(double));
  memset(o->p, 0, cells * sizeof(double));
  const int glz = o->nz;
#pragma omp parallel for schedule(static)
  for (int k = GHOST; k < o->lz - GHOST; ++k)
    for (int j = GHOST; j < o->ly - GHOST; ++j)
      for (int i = GHOST; i < o->lx - GHOST; ++i) {
        const size_t c = C3(o, i, j, k);
        double pm, um, vm, wm;
        moments_ref(&o->f[Q * c], &pm, &um, &vm, &wm);
        if (o->kase == ORACLE_CAVITY) {
          o->p[c] = pm;
          o->ua[c] = um;
          o->va[c] = vm;
          o->wa[c] = wm;
        } else {
          const int s = o->usr[c];
          o->ua[c] = um * s;
          o->va[c] = vm * s;
          o->wa[c] = wm * s;
          o->p[c] = pm * s;
        }
      }
  if (o->kase == ORACLE_CAVITY) {
    /* :343-344: lid velocity forced to 0.1 on the top interior plane */
    for (int j = GHOST; j < o->ly - GHOST; ++j)
      for (int i = GHOST; i < o->lx - GHOST; ++i) o->ua[C3(o, i, j, o->le[2] - 1)] = 0.1;
  } else {
    /* sphere/src/lbm.cpp:403-412: parabolic inlet velocity on x = 3, zero
     * pressure on x = lx - 4 */
    const double u0 = o->u0;
    for (int k = GHOST; k < o->lz - GHOST; ++k)
      for (int j = GHOST; j < o->ly - GHOST; ++j) {
        const size_t c = C3(o, GHOST, j, k);
        o->ua[c] = u0 * 4.0 * (0 + k - GHOST) * (glz - 1 - (0 + k - GHOST)) / ((double)(glz - 1) * (double)(glz - 1));
        o->va[c] = 0.0;
        o->wa[c] = 0.0;
        o->p[C3(o, o->lx - GHOST - 1, j, k)] = 0.0;
      }
  }
}

void oracle_step(oracle_lbm* o, int nsteps) {
  for (int it = 0; it < nsteps; ++it) {
    oracle_collision(o);
    oracle_halo(o);
    oracle_streaming(o);
    oracle_update(o);
  }
}

void oracle_get_moments(const oracle_lbm* o, double* u, double* v, double* w, double* p) {
  for (int k = 0; k < o->nz; ++k)
    for (int j = 0; j < o->ny; ++j)
      for (int i = 0; i < o->nx; ++i) {
        const size_t d = (size_t)i + (size_t)o->nx * ((size_t)j + (size_t)o->ny * k);
        const size_t c = C3(o, i + GHOST, j + GHOST, k + GHOST);
        if (u) u[d] = o->ua[c];
        if (v) v[d] = o->va[c];
        if (w) w[d] = o->wa[c];
        if (p) p[d] = o->p[c];
      }
}

void oracle_get_f(const oracle_lbm* o, double* f) {
  memcpy(f, o->f, (size_t)o->lx * o->ly * o->lz * Q * sizeof(double));
}
void oracle_get_usr(const oracle_lbm* o, int* usr) {
  memcpy(usr, o->usr, (size_t)o->lx * o->ly * o->lz * sizeof(int));
}
void oracle_extents(const oracle_lbm* o, int* lx, int* ly, int* lz) {
  *lx = o->lx;
  *ly = o->ly;
  *lz = o->lz;
}

void oracle_system(int kase, double rho0, double R, int Re, double u0, int time_in, int inter_in, int sx,
                   double* tau, double* miu, double* Ma, int* time_out, int* inter_out) {
  const double cs2 = 1.0 / 3.0, cs = sqrt(cs2);
  *Ma = u0 / cs;
  if (kase == ORACLE_TGV) { /* tgv/src/System.cpp:17-21 */
    *time_out = 100;
    *inter_out = 10;
    *miu = rho0 * u0 * sx / 2 / 3.1415926 / Re;
    *tau = u0 * sx / Re / cs2 / 2 / 3.1415926;
  } else { /* lid_driven_cavity/src/System.cpp:17-19 */
    *miu = rho0 * u0 * R / Re;
    *tau = u0 * R / Re / cs2;
    *time_out = time_in;
    *inter_out = inter_in;
    if (kase == ORACLE_SPHERE) { /* sphere/src/System.cpp:21-22 */
      *time_out = (int)(pow(2 * R, 2) / *miu);
      *inter_out = 1;
    }
  }
}

/* tgv/src/lbm.cpp:335-669 at one rank: 332-byte #!TDV112 header, then x, y,
 * z, u, v, w, p as FP64 arrays with x fastest. */
int oracle_write_tecplot(const oracle_lbm* o, const char* path, int n) {
  FILE* fp = fopen(path, "wb");
  if (!fp) return 1;
  const size_t N = (size_t)o->nx * o->ny * o->nz;
  double* fld[4];
  for (int a = 0; a < 4; ++a) fld[a] = (double*)malloc(N * sizeof(double));
  oracle_get_moments(o, fld[0], fld[1], fld[2], fld[3]);
  double mn[4], mx[4];
  for (int a = 0; a < 4; ++a) {
    mn[a] = 1.7976931348623157e308;
    mx[a] = -1.7976931348623157e308;
    for (size_t c = 0; c < N; ++c) {
      if (fld[a][c] > mx[a]) mx[a] = fld[a][c];
      if (fld[a][c] < mn[a]) mn[a] = fld[a][c];
    }
  }
  int32_t iv;
  float fv;
  double dv;
#define WI(x) (iv = (x), fwrite(&iv, 4, 1, fp))
#define WF(x) (fv = (x), fwrite(&fv, 4, 1, fp))
#define WD(x) (dv = (x), fwrite(&dv, 8, 1, fp))
  fwrite("#!TDV112", 1, 8, fp);
  WI(1);
  WI(0);
  WI(0);
  WI(7);
  const int names[7] = {'x', 'y', 'z', 'u', 'v', 'w', 'p'};
  for (int a = 0; a < 7; ++a) {
    WI(names[a]);
    WI(0);
  }
  WF(299.0f);
  const char* zone = "ZONE 001";
  for (int a = 0; zone[a]; ++a) WI(zone[a]);
  WI(0);
  WI(-1);
  WD((double)n);
  WI(0);
  WI(-1);
  WI(0);
  WI(0);
  WI(0);
  WI(0);
  WI(o->nx);
  WI(o->ny);
  WI(o->nz);
  WI(0);
  WF(357.0f);
  WF(299.0f);
  for (int a = 0; a < 7; ++a) WI(2);
  WI(0);
  WI(0);
  WI(-1);
  WD(0.0);
  WD(1.0);
  WD(0.0);
  WD(1.0);
  WD(0.0);
  WD(1.0);
  for (int a = 0; a < 4; ++a) {
    WD(mn[a]);
    WD(mx[a]);
  }
#undef WI
#undef WF
#undef WD
  double* buf = (double*)malloc(N * sizeof(double));
  for (int axis = 0; axis < 3; ++axis) {
    const int gl = axis == 0 ? o->nx : (axis == 1 ? o->ny : o->nz);
    for (int k = 0; k < o->nz; ++k)
      for (int j = 0; j < o->ny; ++j)
        for (int i = 0; i < o->nx; ++i) {
          const int c = axis == 0 ? i : (axis == 1 ? j : k);
          buf[(size_t)i + (size_t)o->nx * ((size_t)j + (size_t)o->ny * k)] = (double)(0 + c) / (gl - 1);
        }
    fwrite(buf, sizeof(double), N, fp);
  }
  for (int a = 0; a < 4; ++a) fwrite(fld[a], sizeof(double), N, fp);
  free(buf);
  for (int a = 0; a < 4; ++a) free(fld[a]);
  return fclose(fp) == 0 ? 0 : 1;
}

/* ======================================================================
 * Standard-boundary variants (see imexlb_oracle.h).  Interior-only storage,
 * two buffers, the fused order pull -> moments -> collide, FP64 with the
 * reference's expression order (the device's EXACT arithmetic).
 * ====================================================================== */
struct oracle_std {
  int kase, nx, ny, nz;
  double tau0, rho0, u0, lid_u, inlet_u;
  double *A, *B; /* post-collision distributions, index q + Q*cell */
  double *u, *v, *w, *p;
  unsigned char* fluid;
  double feq_in[Q];
  double drag[3];
};

static inline size_t SC(const oracle_std* o, int i, int j, int k) {
  return (size_t)i + (size_t)o->nx * ((size_t)j + (size_t)o->ny * (size_t)k);
}

/* Post-collision populations of one cell from its pulled populations: the
 * reference's moments (moments_ref), equilibrium (feq_tab) and collision
 * (collide_ref), so that only the link rules of oracle_std_step are new. */
static void std_update_cell(const oracle_std* o, const double* f, double* u, double* v, double* w, double* p,
                            double* out) {
  moments_ref(f, p, u, v, w);
  for (int q = 0; q < Q; ++q) out[q] = collide_ref(f[q], feq_tab(q, *u, *v, *w, *p), o->tau0);
}

oracle_std* oracle_std_create(int kase, int nx, int ny, int nz, double tau0, double rho0, double u0,
                              double lid_u, double inlet_u, double sphere_d, double cx, double cy, double cz) {
  if ((kase != ORACLE_CAVITY && kase != ORACLE_SPHERE && kase != ORACLE_SLAB) || nx < 2 || ny < 2 || nz < 2)
    return NULL;
  oracle_std* o = (oracle_std*)calloc(1, sizeof(oracle_std));
  o->kase = kase;
  o->nx = nx;
  o->ny = ny;
  o->nz = nz;
  o->tau0 = tau0;
  o->rho0 = rho0;
  o->u0 = u0;
  o->lid_u = lid_u;
  o->inlet_u = inlet_u;
  const size_t n = (size_t)nx * ny * nz;
  o->A = (double*)calloc(n * Q, sizeof(double));
  o->B = (double*)calloc(n * Q, sizeof(double));
  o->u = (double*)calloc(n, sizeof(double));
  o->v = (double*)calloc(n, sizeof(double));
  o->w = (double*)calloc(n, sizeof(double));
  o->p = (double*)calloc(n, sizeof(double));
  o->fluid = (unsigned char*)malloc(n);
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const size_t c = SC(o, i, j, k);
        int solid = 0;
        if (kase == ORACLE_SPHERE) {
          const double dx = i - cx, dy = j - cy, dz = k - cz;
          solid = dx * dx + dy * dy + dz * dz <= 0.25 * sphere_d * sphere_d;
        }
        o->fluid[c] = (unsigned char)!solid;
        o->u[c] = (kase == ORACLE_SPHERE && !solid) ? inlet_u : 0.0;
      }
  /* the inlet's equilibrium: the reference's feq of (inlet_u, 0, 0) at p = 0 */
  for (int q = 0; q < Q; ++q) o->feq_in[q] = feq_tab(q, inlet_u, 0.0, 0.0, 0.0);
  /* f = feq of the initial fields (tgv/src/lbm.cpp:209-218); the first
   * collision leaves it unchanged */
  for (size_t c = 0; c < n; ++c)
    for (int q = 0; q < Q; ++q) o->A[q + Q * c] = feq_tab(q, o->u[c], o->v[c], o->w[c], o->p[c]);
  return o;
}

void oracle_std_destroy(oracle_std* o) {
  if (!o) return;
  free(o->A);
  free(o->B);
  free(o->u);
  free(o->v);
  free(o->w);
  free(o->p);
  free(o->fluid);
  free(o);
}

void oracle_std_step(oracle_std* o, int nsteps) {
  const int nx = o->nx, ny = o->ny, nz = o->nz;
  for (int s = 0; s < nsteps; ++s) {
    double fx = 0.0, fy = 0.0, fz = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : fx, fy, fz)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          const size_t c = SC(o, i, j, k);
          double f[Q];
          if (o->kase == ORACLE_SPHERE && !o->fluid[c]) {
            o->u[c] = o->v[c] = o->w[c] = o->p[c] = 0.0;
            continue;
          }
          for (int q = 0; q < Q; ++q) {
            const int ex = E_REF[q][0], ey = E_REF[q][1], ez = E_REF[q][2];
            int si = i - ex, sj = j - ey, sk = k - ez;
            if (o->kase == ORACLE_CAVITY || o->kase == ORACLE_SLAB) {
              if (o->kase == ORACLE_SLAB) {
                si = (si + nx) % nx;
                sj = (sj + ny) % ny;
              }
              if (si >= 0 && si < nx && sj >= 0 && sj < ny && sk >= 0 && sk < nz) {
                f[q] = o->A[q + Q * SC(o, si, sj, sk)];
              } else {
                double val = o->A[BB_REF[q] + Q * c];
                if (ex != 0 && sk >= nz) val += ((6.0 * o->rho0) * o->lid_u) * W_REF[q] * (double)ex;
                f[q] = val;
              }
            } else {
              sj = (sj + ny) % ny;
              sk = (sk + nz) % nz;
              if (si < 0) {
                f[q] = o->feq_in[q];
              } else {
                if (si >= nx) si = nx - 1;
                const size_t sc = SC(o, si, sj, sk);
                if (!o->fluid[sc]) {
                  f[q] = o->A[BB_REF[q] + Q * c];
                  fx += -2.0 * f[q] * ex;
                  fy += -2.0 * f[q] * ey;
                  fz += -2.0 * f[q] * ez;
                } else {
                  f[q] = o->A[q + Q * sc];
                }
              }
            }
          }
          std_update_cell(o, f, &o->u[c], &o->v[c], &o->w[c], &o->p[c], &o->B[Q * c]);
        }
    double* t = o->A;
    o->A = o->B;
    o->B = t;
    o->drag[0] = fx;
    o->drag[1] = fy;
    o->drag[2] = fz;
  }
}

void oracle_std_get_moments(const oracle_std* o, double* u, double* v, double* w, double* p) {
  const size_t n = (size_t)o->nx * o->ny * o->nz;
  if (u) memcpy(u, o->u, n * sizeof(double));
  if (v) memcpy(v, o->v, n * sizeof(double));
  if (w) memcpy(w, o->w, n * sizeof(double));
  if (p) memcpy(p, o->p, n * sizeof(double));
}

void oracle_std_drag(const oracle_std* o, double* fx, double* fy, double* fz) {
  *fx = o->drag[0];
  *fy = o->drag[1];
  *fz = o->drag[2];
}

/* Check of the three-operation correctly rounded division by 3 the device's
 * EXACT mode uses for the moments: returns how many of n random doubles
 * (random signs, exponents in [-200, 200] around 1, random significands)
 * give a quotient different from IEEE division.  planted = 1 drops the
 * correction step (q0 = x * RN(1/3) alone), a known-wrong variant that shows
 * the check can fail. */
int oracle_check_div3(long n, unsigned long long seed, int planted) {
  const double z = 0x1.5555555555555p-2;
  int bad = 0;
  unsigned long long s = seed ? seed : 88172645463325252ULL;
  for (long t = 0; t < n; ++t) {
    s ^= s << 13;
    s ^= s >> 7;
    s ^= s << 17;
    const unsigned long long mant = s & 0xFFFFFFFFFFFFFULL;
    const long e = (long)((s >> 52) % 401) - 200;
    const unsigned long long sign = (s >> 63) << 63;
    union {
      unsigned long long u;
      double d;
    } v;
    v.u = sign | ((unsigned long long)(1023 + e) << 52) | mant;
    const double x = v.d;
    const double q0 = x * z;
    const double r = fma(-q0, 3.0, x);
    const double q1 = planted ? q0 : fma(r, z, q0);
    if (q1 != x / 3.0) ++bad;
  }
  return bad;
}

/* Check of the EXACT mode's collision division (kernels' div_rn): x/d by
 * Markstein's correction with an exactness test and IEEE division for the
 * cases the test rejects.  n random x (random signs, exponents within 2^+-60,
 * random significands) against random divisors d in [0.5, 4) (a fresh d every
 * 1024 samples; every 997th x is zero and every 1009th tiny, which the
 * exactness test rejects on purpose).  Returns the number of quotients that
 * differ from x / d; *fallbacks counts the rejected cases.  planted = 1
 * returns the uncorrected q0 = RN(x RN(1/d)) (a known-wrong variant). */
int oracle_check_div(long n, unsigned long long seed, int planted, long* fallbacks) {
  unsigned long long s = seed ? seed : 0x9E3779B97F4A7C15ULL;
  int bad = 0;
  long fb = 0;
  double d = 1.0, z = 1.0;
  for (long t = 0; t < n; ++t) {
    s ^= s << 13;
    s ^= s >> 7;
    s ^= s << 17;
    union {
      unsigned long long u;
      double v;
    } cv;
    if ((t & 1023) == 0) {
      cv.u = (1023ULL << 52) | (s & 0xFFFFFFFFFFFFFULL);
      d = cv.v * (double)(1u << ((s >> 60) & 1)) * 0.5 * (((s >> 61) & 1) ? 4.0 : 1.0);
      if (d >= 4.0) d *= 0.5;
      z = 1.0 / d;
      s ^= s << 13;
      s ^= s >> 7;
      s ^= s << 17;
    }
    const long e = (t % 1009 == 0) ? -1000 : (long)((s >> 52) % 121) - 60;
    cv.u = ((s >> 63) << 63) | ((unsigned long long)(1023 + e) << 52) | (s & 0xFFFFFFFFFFFFFULL);
    double x = (t % 997 == 0) ? ((t & 1) ? -0.0 : 0.0) : cv.v; /* zeros of both signs */
    if (t % 1013 == 0) x = (t & 1) ? -INFINITY : INFINITY;
    if (t % 1019 == 0) x = NAN;
    const double q0 = x * z;
    const double r0 = fma(-q0, d, x);
    const double q1 = fma(r0, z, q0);
    const double r1 = fma(-q1, d, x);
    union {
      double v;
      unsigned long long u;
    } qb = {q1};
    /* the device's test on the high word of q1 (step_core.cuh div_rn_fast) */
    const int hi = (int)(qb.u >> 32);
    const int he = (hi & 0x7ff00000) - (53 << 20);
    double q;
    int accept = 0;
    if (he > 0 && (hi & 0x000fffff) != 0) {
      union {
        unsigned long long u;
        double v;
      } hg = {(unsigned long long)(unsigned)he << 32};
      accept = fabs(r1) < d * hg.v;
    }
    if (planted) {
      q = q0;
    } else if (accept) {
      q = q1;
    } else if (x == 0.0 || !isfinite(x)) {
      q = x; /* +-0 / d = +-0, +-inf / d = +-inf for d > 0; NaN stays NaN */
    } else {
      q = x / d;
      ++fb;
    }
    const double want = x / d;
    if (isnan(want) ? !isnan(q) : memcmp(&q, &want, sizeof q) != 0) ++bad; /* bit patterns: a zero's sign counts */
  }
  if (fallbacks) *fallbacks = fb;
  return bad;
}
