/* CPU oracle for the CosTuuM T-matrix hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference algorithms (CosTuuM, header-only
 * C++), written so that every step keeps the reference's operation order.
 * It is the checker for the CUDA path: only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg may load it. Parity of this oracle is pinned
 * against the unmodified reference (oracle/build_ref.sh) by the golden
 * fixtures in tests/golden/ and by the reference's own Mishchenko fixture.
 *
 * Complex arrays are interleaved (re, im) doubles in every signature.
 * Block storage of a T-matrix follows the reference's index map
 * (src/TMatrixResource.hpp:195-213): block m has size 2nb x 2nb, nb = nmax for
 * m = 0 and nmax + 1 - m for m >= 1; row (i, n) -> i*nb + n - max(m, 1).
 */
#ifndef TMX_ORACLE_H
#define TMX_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* special functions (src/SpecialFunctions.hpp) */
void or_gauss_legendre(int order, double *x, double *w);
void or_gauss_legendre_ab(int order, double a, double b, double *x, double *w);
void or_bessel_j_real(int nmax, double z, double *j, double *dj);
void or_bessel_y_real(int nmax, double z, double *y, double *dy);
void or_bessel_j_complex(int nmax, double zr, double zi, double *j, double *dj);
/* the same recurrences started at index `start` instead of 800 */
void or_bessel_j_real_start(int nmax, int start, double z, double *j,
                            double *dj);
void or_bessel_j_complex_start(int nmax, int start, double zr, double zi,
                               double *j, double *dj);
void or_wigner_d(double cosx, int nmax, int m, double *d, double *dd);
void or_wigner_d_sinx(double cosx, double sinx, double sinx_inv, int nmax,
                      int m, double *d, double *dd);
double or_rv_over_rs(double axis_ratio);
int or_clebsch_gordan_row(int n1, int n2, int N, double *C);

/* dense complex inverse (src/Matrix.hpp:261-384), row major n x n */
void or_plu_inverse(int n, double *a);

/* orientation distribution expansion coefficients p_0..p_order
 * kind 0: random (numerical quadrature), 1: Mishchenko (param = cos2beta),
 * 2: Davis-Greenstein (param = axis ratio) */
void or_orientation_coefficients(int kind, double param, int order,
                                 double *out);

/* number of doubles (2 x complex count) of a full T-matrix up to nmax */
long or_tmatrix_size(int nmax);
long or_tmatrix_block_offset(int nmax, int m);

/* one order of the m = 0 convergence chain (TMatrixM0Task::execute):
 * writes T0 (2 nmax x 2 nmax complex) and the m = 0 sums */
void or_tmatrix_m0(double r_ev, double wavelength, double mr, double mi,
                   double axis_ratio, int nmax, int ngauss, double *T0,
                   double *qsca, double *qext);

/* block m >= 1 at converged (nmax, ngauss) (TMatrixMAllTask::execute) */
void or_tmatrix_mblock(double r_ev, double wavelength, double mr, double mi,
                       double axis_ratio, int nmax, int ngauss, int m,
                       double *Tm);

/* full task-based computation of one grain: convergence chain over orders
 * min_order .. max_order - 1 (TaskManager.hpp:1146-1197) then all m blocks.
 * T must hold or_tmatrix_size(max_order) doubles. info[0..5] =
 * {chain Qsca, chain Qext, full Qsca, full Qext, dQs, dQe}.
 * Returns nmax; *ngauss and *converged are set. */
int or_tmatrix_converge(double r_ev, double wavelength, double mr, double mi,
                        double axis_ratio, int min_order, int max_order,
                        int glfac, double tolerance, double *T, int *ngauss,
                        int *converged, double *info);

/* TMatrixQTask (TMatrixResource.hpp:1136-1210): full Qsca, Qext sums */
void or_tmatrix_q(int nmax, const double *T, double *qsca, double *qext);

/* AlignmentAverageTask (AlignmentAverageTask.hpp:115-215); coeffs holds the
 * expansion coefficients p_0 .. p_{2 nmax}; coeffs == NULL copies T */
void or_orientation_average(int nmax, const double *T, const double *coeffs,
                            double *Tavg);

/* ExtinctionCoefficientTask::execute: out[3 * ntheta] = Qext, Qextpol,
 * Qextcpol per angle */
void or_extinction(int nmax, const double *T, double wavelength, double r_ev,
                   int ntheta, const double *theta, double *out);

/* AbsorptionCoefficientTask::execute: out[2 * ntheta] = Qabs, Qabspol */
void or_absorption(int nmax, const double *T, double wavelength, double r_ev,
                   int ntheta, const double *theta, int ngauss,
                   int account_for_scattering, double *out);

/* ScatteringMatrixTask::execute on the get_table grid (theta_in = pi/2,
 * ntheta GL zenith, 2 ntheta GL azimuth): out[ntheta * 2 ntheta * 16] */
void or_scattering_matrix(int nmax, const double *T, double wavelength,
                          int ntheta, double *out);

/* plain path: TMatrixCalculator::calculate_TMatrix orders
 * (TMatrixCalculator.hpp:64-213); returns 1 where the reference aborts */
int or_calculator_orders(double r_ev, double wavelength, double mr, double mi,
                         double axis_ratio, int maximum_order, double tolerance,
                         int ndgs, int maximum_ngauss, int *nmax, int *ngauss);

/* lab-frame amplitude matrix S (2 x 2 complex, interleaved) at particle
 * orientation (alpha, beta) (TMatrix.hpp:1109-1460) */
void or_amplitude_lab(int nmax, const double *T, double wavelength, double alpha,
                      double beta, double theta_in, double phi_in,
                      double theta_out, double phi_out, double *S);

/* Z (TMatrix.hpp:1896-1948) and K (:1972-2010) from S, row major 4 x 4 */
void or_z_from_s(const double *S, double *Z);
void or_k_from_s(double wavelength, const double *S, double *K);

#ifdef __cplusplus
}
#endif

#endif
