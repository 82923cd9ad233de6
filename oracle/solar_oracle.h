/*
 * solar_oracle.h -- C API of the FP64 CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker and the timed CPU
 * baseline for the GPU solver.  Only the test suite, the smoke check and the
 * benchmark's CPU-baseline / reference arm may load it; the product never links it.
 *
 * The oracle restates, loop by loop and in double precision, the time-stepping path
 * of the cubed-sphere acoustic solver ankitvb/solar (Fortran 90 + MPI) with all six
 * faces held in one process (the reference's px = py = pr = 1 case).  Every function
 * cites the reference routine it follows.
 *
 * Parity status: UNPINNED against golden vectors.  The reference ships no golden
 * vectors or tolerance tests, and it cannot be built here (no Fortran compiler, no
 * MPI).  The oracle is instead pinned to the reference's own analytic print-checks
 * (testcode.f90:53-303), turned into assertions in tests/test_oracle_kat.py.
 *
 * Array conventions: a "field" array holds all six faces,
 *   f[zone][k][j][i]        (zone 0..5, k radial 0..nr-1, j eta, i xi; i fastest)
 * which is the reference's per-zone Fortran array f(mx,my,mr) concatenated in zone
 * order.  The state q holds five fields per zone, exactly COMMON /RKWORK/ q(mx,my,mr,5):
 *   q[zone][m][k][j][i]     (m = rho, v_xi, v_eta, v_r, p)
 */
#ifndef SOLAR_ORACLE_H
#define SOLAR_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_ctx oracle_ctx;

/* model: nr rows of 8 columns, row-major, as the file 'solar_model' is read at
 * ic_acoustic_wave.f90:61-67 (r/R, c, rho, p, T, g, Gamma, unused).
 * c2_3d: optional per-point c^2 (field layout), replacing the radial c^2 after the
 * SOLAR_DATA normalisation; NULL for the reference's radial background.
 * Sponge settings mirror sponge.f90:20-29 (a_sponge, s_exp, k_sponge_length) plus two
 * switches that keep the lower / upper branch of sponge.f90:40-46. */
oracle_ctx* oracle_create(int nx, int nr, const double* model, double dt,
                          double a_sponge, double s_exp, int k_sponge_length,
                          int sponge_lower, int sponge_upper, const double* c2_3d);
void oracle_destroy(oracle_ctx* c);
/* 0 (default): reference arithmetic.  1: on the eight inter-zone vector strips that the
 * receiver reverses, evaluate the receiver-frame rotation (transform.f90:184-274) at the
 * mirrored edge index instead of the sender's own index. */
void oracle_set_fix_reversed_rotation(oracle_ctx* c, int on);
void oracle_set_threads(int n);

/* Grid queries: which = 0 theta, 1 phi (6*nx*nx each), 2 gxi (nx), 3 gr (nr),
 * 4 gdrdchi (nr), 5 interpolant (3*nx*9, [layer][point][iter+4]), 6 interpoints
 * (3*nx), 7 c2 (nr), 8 rho0 (nr), 9 g0 (nr), 10 sigma_r (nr), 11 drho0dr (nr) */
int oracle_get_grid(const oracle_ctx* c, int which, double* out);

/* Gaussian pressure pulse p = amp*exp(-|x-x0|^2/(2 w^2)) added to field 5, with
 * x = r (sin th cos ph, sin th sin ph, cos th) from the reference's own theta, phi
 * (metric.f90:97-158). */
void oracle_add_gaussian(const oracle_ctx* c, double* q, double x0, double y0, double z0,
                         double width, double amp);

/* Operators (single field arrays, six zones) */
void oracle_interpolate_strips(const oracle_ctx* c, const double* f, double* strips);
    /* strips[zone][edge S,N,W,E][k][layer][t] -- INTERPOLATE_ALONG_X/Y of the four edge
       strips (grad.f90:187-190) */
void oracle_ddx(const oracle_ctx* c, const double* f, double* out);   /* scalar halos */
void oracle_ddy(const oracle_ctx* c, const double* f, double* out);
void oracle_ddr(const oracle_ctx* c, const double* f, double* out);
void oracle_gradient(const oracle_ctx* c, const double* p, double* gxi, double* geta,
                     double* gr);
void oracle_divergence(const oracle_ctx* c, const double* vxi, const double* veta,
                       const double* vr, double* div);
void oracle_filter_field(const oracle_ctx* c, const double* f, double* out, int which);
    /* which: 0 = FILTER_XI, 1 = FILTER_ETA (halos from f), 2 = FILTER_R */

/* Physics plug-ins and the time step (state arrays) */
void oracle_compute_rhs(const oracle_ctx* c, const double* q, double* rhs);
void oracle_bc_rhs(const oracle_ctx* c, double* rhs);
void oracle_sponge(const oracle_ctx* c, const double* q, double* rhs);
void oracle_filter_exp(const oracle_ctx* c, const double* q, double* qf);
void oracle_rk4(const oracle_ctx* c, double* q, int nsteps);
double oracle_norm(const oracle_ctx* c, const double* q, int field);

/* COMPUTE_CURL (grad.f90:140-255) with TRANSFORM_VECTOR_BETWEEN_MESHES_CURL
 * (transform.f90:279-498): (a_xi, a_eta, a_r) -> (curl_xi, curl_eta, curl_r), six-zone fields. */
void oracle_curl(const oracle_ctx* c, const double* axi, const double* aeta, const double* ar, double* cxi,
                 double* ceta, double* cr);

/* Source term of the v_r equation (compute_rhs_acoustic.f90:92-116): kind 0 off, 1 analytic
 * with centre plane k_center (0-based), 2 sampled S_t (LAGRANGE_INTERP) at plane e_rad;
 * nstep = the run's step count.  Samples in READ_FORCING_FUNC order f[(i*nx + j)*nt + n].
 * The clock (time, step) starts at 0 and RK4 advances it. */
int oracle_set_forcing(oracle_ctx* c, int kind, int k_center, int nstep);
int oracle_set_forcing_samples(oracle_ctx* c, int zone, const double* f, int nt);
void oracle_set_clock(oracle_ctx* c, double time, int step);
void oracle_get_clock(const oracle_ctx* c, double* time, int* step);

#ifdef __cplusplus
}
#endif
#endif
