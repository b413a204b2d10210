/* CPU restatement of the imexlb proxy apps' D3Q27 lattice-Boltzmann step.
 *
 * TEST INFRASTRUCTURE ONLY: the parity tests, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py use it as the checker.  The product path never
 * calls it.
 *
 * Pinning: tests/test_oracle_pinning.py checks this restatement against the
 * reference's own solver sources (compiled by `make -C oracle ref` against the
 * single-rank Kokkos/MPI stand-in in oracle/refshim) and against the golden
 * fixtures in tests/golden that were generated from them.
 *
 * Storage follows the reference: padded extents lx = nx + 6 (ghost = 3,
 * tgv/src/lbm.hpp:22, :168-170), distributions f(ii, i, j, k) with the
 * population index fastest (Kokkos LayoutLeft of a CudaUVMSpace view,
 * tgv/src/lbm.hpp:149), scalar fields (i, j, k) with i fastest.
 */
#ifndef IMEXLB_ORACLE_H
#define IMEXLB_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { ORACLE_TGV = 0, ORACLE_CAVITY = 1, ORACLE_SPHERE = 2, ORACLE_SLAB = 3 };

typedef struct oracle_lbm oracle_lbm;

/* Parameters as the reference's LBM constructor receives them
 * (tgv/src/lbm.hpp:161): interior extents, tau0 (= 3 nu), rho0, u0.
 * ran_padded (lx*ly*lz ints, i fastest) is the sphere's random field; it may
 * be NULL (zeros). */
oracle_lbm* oracle_create(int kase, int nx, int ny, int nz, double tau0, double rho0, double u0,
                          const int* ran_padded);
void oracle_destroy(oracle_lbm* o);

void oracle_initialize(oracle_lbm* o); /* LBM::Initialize */
void oracle_collision(oracle_lbm* o);  /* LBM::Collision */
void oracle_halo(oracle_lbm* o);       /* pack + exchange + unpack at one rank */
void oracle_streaming(oracle_lbm* o);  /* LBM::Streaming (boundary passes + stream) */
void oracle_update(oracle_lbm* o);     /* LBM::Update */
void oracle_step(oracle_lbm* o, int nsteps);

/* interior fields, x fastest (nx*ny*nz) */
void oracle_get_moments(const oracle_lbm* o, double* u, double* v, double* w, double* p);
/* padded state: f is q*lx*ly*lz (population fastest); usr is lx*ly*lz */
void oracle_get_f(const oracle_lbm* o, double* f);
void oracle_get_usr(const oracle_lbm* o, int* usr);
void oracle_extents(const oracle_lbm* o, int* lx, int* ly, int* lz);

/* Parameter derivation of System::System from the nine input.in numbers
 * (tgv/src/System.cpp:12-21, lid_driven_cavity/src/System.cpp:11-19,
 * sphere/src/System.cpp:11-22).  Outputs tau, miu, Ma, Time, inter. */
void oracle_system(int kase, double rho0, double R, int Re, double u0, int time_in, int inter_in, int sx,
                   double* tau, double* miu, double* Ma, int* time_out, int* inter_out);

/* Tecplot binary writer of LBM::MPIoutput at one rank (tgv/src/lbm.cpp:335-669) */
int oracle_write_tecplot(const oracle_lbm* o, const char* path, int n);

/* Mismatches of the device's three-operation x/3 against IEEE division over n
 * random doubles (test of the EXACT-mode moment arithmetic). */
int oracle_check_div3(long n, unsigned long long seed, int planted);

/* Mismatches of the device's checked Markstein division x/d against IEEE
 * division over n random (x, d), d in [0.5, 4); *fallbacks = rejected cases. */
int oracle_check_div(long n, unsigned long long seed, int planted, long* fallbacks);

/* Number of OpenMP threads the oracle will use (for the CPU baseline). */
int oracle_threads(void);

/* ------------------------------------------------------------------------
 * Standard-boundary variants (the BASELINE configurations; no reference
 * code exists for them, so this is the specification the device path is
 * checked against):
 *   ORACLE_CAVITY: fluid box [0,n)^3, halfway bounce-back on all six walls,
 *     the lid (z >= nz) moving along +x at lid_u:
 *       f_q(x) = f*_bb(q)(x) + 6 w_q rho0 (e_q . u_w)   when x - e_q is a wall
 *   ORACLE_SPHERE: channel periodic in y and z, equilibrium inlet
 *     feq(p = 0, u = (inlet_u, 0, 0)) for populations entering at x = 0,
 *     zero-gradient outlet (a population entering at x = nx-1 is pulled
 *     from x = nx-1 instead of x = nx), halfway bounce-back on the voxelised
 *     sphere |x - c|^2 <= d^2/4; solid cells are not updated and report
 *     zero moments.  Drag = sum over links of -2 f_q(x) e_q.
 *   ORACLE_SLAB: the cavity's rules on a slab periodic in x and y: halfway
 *     bounce-back at the bottom (z < 0, at rest) and at the lid (z >= nz,
 *     moving along +x at lid_u); its steady state is plane Couette flow,
 *     u(z) = lid_u (z + 1/2) / nz.
 * All use the reference's moments, equilibrium and collision (feq_tab,
 * moments_ref, collide_ref: the expressions of the reference's Update and
 * Collision, FP64): only the link rules above are this specification's own.
 * ------------------------------------------------------------------------ */
typedef struct oracle_std oracle_std;
oracle_std* oracle_std_create(int kase, int nx, int ny, int nz, double tau0, double rho0, double u0,
                              double lid_u, double inlet_u, double sphere_d, double cx, double cy, double cz);
void oracle_std_destroy(oracle_std* o);
void oracle_std_step(oracle_std* o, int nsteps);
void oracle_std_get_moments(const oracle_std* o, double* u, double* v, double* w, double* p);
/* momentum-exchange force of the last step (sphere channel) */
void oracle_std_drag(const oracle_std* o, double* fx, double* fy, double* fz);


#ifdef __cplusplus
}
#endif
#endif
