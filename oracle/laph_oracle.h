/*
 * laph_oracle.h -- CPU FP64 oracle for the per-timeslice LapH eigensystem path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library restates, on the CPU and in plain
 * C++17 + OpenMP, the algorithms of HISKP-LQCD/LapH_EigSys that the B200
 * library (laph_eigsys_b200) re-implements.  Only the tests, the smoke check
 * and bench.py's CPU-baseline leg may load it, and only as the checker or the
 * timed CPU baseline -- never as a product code path.
 *
 * Parity status: the arithmetic is UNPINNED against reference outputs.  The
 * reference cannot be built here as a whole (Eigen, PETSc, SLEPc, c-lime,
 * Boost and MPI are absent) and it ships no golden vectors, stored eigenvalues
 * or fixtures.  Its parameter parser and lookup tables (modules/par_io.cpp,
 * modules/navigation.cpp) need only the standard library; the tests compile
 * them unchanged into a driver (oracle/_ref/ref_dump) and check this oracle's
 * site indexing, matvec, smearings, source shape and displacement against the
 * reference's formulas evaluated on those compiled tables.  Beyond that the
 * oracle is pinned by analytic known answers that follow from the reference's
 * own checks: the unit gauge field (free spectrum sum_i 4 sin^2(pi n_i / L)
 * with its degeneracies), pure-gauge fields (gauge-covariant spectrum), SU(3)
 * unitarity/determinant, tr(V^dag V) = nev, and a dense eigendecomposition of
 * the assembled operator for small L.
 *
 * Conventions (all follow the reference):
 *   site   = x*L*L + y*L + z                         (modules/navigation.cpp:27-88)
 *   links3 = double[V3][3 dirs][3][3][re,im], row-major 3x3, dir 0/1/2 = x/y/z
 *            (Tslice::eigen_timeslice, modules/timeslice.cpp:34-79)
 *   conf   = double[nt][V3][4 slots][3][3][re,im], slot 0 = U_t, 1..3 = U_x..U_z
 *            (read_lime_gauge_field_doubleprec_timeslices, modules/io.cpp:112-131)
 *   vector = complex128[3*V3], index 3*site + colour  (modules/shell_matop.cpp:33-38)
 *   eigensystem = complex128 column-major [3*V3][nev] (src/ev_ts.cpp:298)
 */
#ifndef LAPH_ORACLE_H_
#define LAPH_ORACLE_H_
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

void orc_set_threads(int n);

/* LIME/ILDG reader restating modules/io.cpp:22-146.  Returns 0 on success,
 * 500 open/read error, -2 no ildg-binary-data record, 501 wrong size,
 * 502 single-precision file (the reference prints "Not implemented"). */
int orc_lime_read_gauge(const char* path, int T, int L, int t_i, int t_f, double* conf);

/* Tslice::map_timeslice_to_eigen (modules/timeslice.cpp:34-79). */
void orc_map_timeslice(const double* conf_ts, int L, double* links3);

/* proj_to_su3_imp (modules/timeslice.cpp:90-104): W = M (M^dag M)^{-1/2},
 * then W * det(W)^{-1/3} with the principal complex cube root. In place. */
void orc_proj_su3(double* m18);

/* exp(i*H) for a Hermitian 3x3 H (used for exp(-q) of smearing_stout). */
void orc_expiH(const double* h18, double* out18);

/* Smearings of modules/timeslice.cpp.  compat=1 keeps the reference's
 * backward-staple factor U[nu][dir] (timeslice.cpp:171-172, :221-222);
 * compat=0 uses the gauge-covariant U[nu][not_dir]. */
void orc_smear_stout(double* links3, int L, double rho, int iter, int compat);
void orc_smear_ape(double* links3, int L, double alpha, int iter, int compat);
void orc_smear_hyp(double* links3, int L, double alpha1, double alpha2, int iter);

/* tv2 (modules/shell_matop.cpp:16-103): y = c(hop(x) - 6x) + a x. */
void orc_tv2(const double* links3, int L, double lam_l, double lam_c, const double* x, double* y);
/* tv_iter (modules/shell_matop.cpp:136-168): y = T_deg(B) x; deg <= 1 leaves y unwritten. */
void orc_tv_iter(const double* links3, int L, double lam_l, double lam_c, int deg, const double* x, double* y);
/* y = (-Delta) x = 6x - hop(x). */
void orc_neglap(const double* links3, int L, const double* x, double* y);
/* Average spatial plaquette (modules/config_utils.cpp:388-426). */
double orc_plaquette(const double* links3, int L);

/* Restarted Krylov-Schur (thick-restart Lanczos, full reorthogonalisation) on
 * the Hermitian operator T_deg(B), largest magnitude -- the SLEPc EPS set-up
 * of src/ev_ts.cpp:231-263.  theta_out[nev] are eigenvalues of T_deg(B)
 * sorted by decreasing |theta|; V_out is column-major complex [3*V3][nev].
 * Convergence: |beta_m s_{m,i}| <= tol*|theta_i| (SLEPc's relative test).
 * ncv <= 0 selects SLEPc's default max(2*nev, nev+15).  Returns 0 when nev
 * pairs converged, 1 when max_it was reached (pairs still returned). */
int orc_eps_solve(const double* links3, int L, double lam_l, double lam_c, int deg,
                  int nev, int ncv, double tol, int max_it, uint64_t seed,
                  double* theta_out, double* V_out, int* nconv_out, int* its_out,
                  long long* nmatvec_out);

/* recover_spectrum (modules/recover_spec.cpp:13-54). */
void orc_recover_spectrum(int nev, const double* theta, int deg, double lam_l, double lam_c, double* out);
/* fix_phase (modules/eigensystem.cpp:4-30). */
void orc_fix_phase(int dim, int nev, const double* V, double* Vfix, double* phase);
/* reset_phase (modules/eigensystem.cpp:32-57): first entry of column n rotated to phase_want[n]. */
void orc_reset_phase(int dim, int nev, const double* V, const double* phase_want, double* Vreset);

/* Dense Hermitian matrix of -Delta (BuildLaplacian analogue,
 * modules/config_utils.cpp:18-58), complex128 row-major [dim][dim]. */
void orc_build_neglap_dense(const double* links3, int L, double* A);

/* right_displacement_one_dir (modules/config_utils.cpp:344-382) on the
 * column-major complex128 block V [3*V3][nev] -> W, links3 as above. */
void orc_displace(const double* links3, int L, int dir, const double* V, int nev, double* W);

/* Source shape psi(r) (modules/sourceshape_funcs.cpp:30-81) on the grid
 * r_i = 0, 2, ... < L, r1 outer and r3 inner: psi[(L+1)/2 cubed].  V is the
 * column-major complex128 eigensystem [3*V3][nev]. */
void orc_sourceshape(const double* V, int L, int nev, double* psi);
/* avg_radii (sourceshape_funcs.cpp:100-135); returns the number of radii. */
int orc_sourceshape_avg(int L, const double* psi, double* r_out, double* psi_out);

/* Seeded synthetic gauge field U = exp(i eps H) of the benchmark inputs, all 4
 * links of nt timeslices, [t][site][mu][3][3] complex128 (the ILDG slice
 * layout); same normal stream as the library's laph_gauge_random. */
void orc_gauge_random(double* conf, int L, int nt, double eps, uint64_t seed);

/* Window MLP (16->64->64->3, tanh) mean-squared loss and gradient, FP64. */
double orc_mlp_loss_grad(const double* params, const double* X, const double* Y, int n, double* grad);

#ifdef __cplusplus
}
#endif
#endif
