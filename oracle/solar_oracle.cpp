// solar_oracle.cpp -- FP64 CPU restatement of the ankitvb/solar time-stepping path.
//
// TEST INFRASTRUCTURE ONLY: the parity checker and the timed CPU baseline.  Nothing in
// the product links or loads this file.  Parity is UNPINNED against golden vectors (the
// reference ships none and cannot be built here: there is no Fortran compiler or MPI);
// it is pinned to the reference's own analytic checks (testcode.f90:53-303) instead.
//
// All six cubed-sphere zones live in one process, which is the reference's
// px = py = pr = 1 decomposition: every "intra-zone" MPI exchange of the reference is
// empty and every inter-zone exchange is a copy between zone arrays, routed exactly as
// the MPI_INTERCOMM sends/receives route them.  Loop bodies follow the reference's
// arithmetic order (accumulate into 0.0, left-to-right products) so the oracle is a
// literal restatement rather than an independent discretisation.
//
// Layout: field arrays f[zone][k][j][i] (i fastest), the reference's per-zone Fortran
// f(mx,my,mr) concatenated over zones.  Edge strips s[edge][k][layer][t] with edge order
// S, N, W, E; t runs along the edge (i for S/N, j for W/E), layer 0..2 is the reference's
// noverlap index 1..3.

#include "solar_oracle.h"

#include <cmath>
#include <cstring>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int NST = 3;    // header:25  nst = noverlap = (nstencil-1)/2
constexpr int NORD = 4;   // header:24
constexpr int NSTR = 5;   // header:26
constexpr int NSTENCIL = 7;
const double PI = std::acos(-1.0);  // header:148

// header:40-46, Tam & Webb DRP first-derivative stencil, index iter+3.
const double COEFFS1[7] = {-0.02651995, 0.18941314, -0.79926643, 0.0,
                           0.79926643, -0.18941314, 0.02651995};
// header:49-55, Tam & Dong one-sided boundary stencils bdy_coeffs1(row, iter); the
// Fortran DATA statement fills the (3,7) array column by column.
const double BDY1[3][7] = {
    {-2.192280339, 4.748611401, -5.108851915, 4.461567104, -2.833498741, 1.128328861,
     -0.203876371},
    {-0.209337622, -1.084875676, 2.147776050, -1.388928322, 0.768949766, -0.28181465,
     0.048230454},
    {0.049041958, -0.468840357, -0.474760914, 1.273274737, -0.518484526, 0.166138533,
     -0.026369431}};
// header:68-76, 2N-storage RK (Cook & Cabot)
const double ALPHA_RK4[5] = {0.0, -4.801594388477952e-01, -1.404247195200064e+00,
                             -2.016477077503357e+00, -1.056444269767207e+00};
const double BETA_RK4[5] = {1.028639988104959e-01, 7.408540575766301e-01,
                            7.426530946683799e-01, 4.694937902357905e-01,
                            1.881733382887932e-01};
// header:99-105, xi/eta filter; header:123-133, radial filter.
const double FILT[7] = {0.015625, -0.09375, 0.234375, 0.6875, 0.234375, -0.09375, 0.015625};
const double FILT_R[11] = {0.0009765, -0.0097655, 0.043945, -0.1171875, 0.2050775, 0.753906,
                           0.2050775, -0.1171875, 0.043945, -0.0097655, 0.0009765};

enum { ES = 0, EN = 1, EW = 2, EE = 3 };

struct Route { int src; int edge; int rev; };
// Inter-zone halo routing for px = py = 1.  For each receiving zone (index 0..5): the
// strip that lands in fp (low side) and fn (high side).
//  xi direction: DDX derivative.f90:374-452 (sends interpol_left=W / right=E of the
//  caller, low/high = transposed S/N), reversal derivative.f90:539-561; FILTER_XI
//  filter.f90:93-171, 257-279 (intended reversal).
const Route ROUTE_X[6][2] = {
    {{3, EE, 0}, {1, EW, 0}},  // zone 1: fp <- zone 4 E (INTERCOMM(1,4)), fn <- zone 2 W
    {{0, EE, 0}, {2, EW, 0}},  // zone 2
    {{1, EE, 0}, {3, EW, 0}},  // zone 3
    {{2, EE, 0}, {0, EW, 0}},  // zone 4
    {{3, EN, 1}, {1, EN, 0}},  // zone 5: fp <- zone 4 N reversed (INTERCOMM(4,5))
    {{3, ES, 0}, {1, ES, 1}},  // zone 6: fn <- zone 2 S reversed (INTERCOMM(2,6))
};
//  eta direction: DDY derivative.f90:55-133, reversal derivative.f90:217-282;
//  FILTER_ETA filter.f90:364-443, 528-593.
const Route ROUTE_Y[6][2] = {
    {{5, EN, 0}, {4, ES, 0}},  // zone 1: fp <- zone 6 N (INTERCOMM(1,6)), fn <- zone 5 S
    {{5, EE, 1}, {4, EE, 0}},  // zone 2: fp <- zone 6 E reversed, fn <- zone 5 E
    {{5, ES, 1}, {4, EN, 1}},  // zone 3: both reversed
    {{5, EW, 0}, {4, EW, 1}},  // zone 4: fn <- zone 5 W reversed
    {{0, EN, 0}, {2, EN, 1}},  // zone 5: fp <- zone 1 N, fn <- zone 3 N reversed
    {{2, ES, 1}, {0, ES, 0}},  // zone 6: fp <- zone 3 S reversed, fn <- zone 1 S
};

}  // namespace

struct oracle_ctx {
  int nx, nr;
  size_t plane, vol;            // nx*nx, nx*nx*nr
  double dxi, deta, dchi, dt;
  std::vector<double> gxi, geta, gchi, gr, gdrdchi;
  std::vector<double> tanxi, taneta, mC, mD;          // per i / j
  std::vector<double> delta, sdelta, XY, CD;          // [j][i]
  std::vector<double> interpoints;                    // [layer][t]
  std::vector<double> interpolant;                    // [layer][t][iter+4]
  std::vector<double> theta, phi;                     // [zone][j][i]
  std::vector<double> c2, rho0, g0, drho0dr, sigma;   // radial
  std::vector<double> c2_3d;                          // optional [zone][k][j][i]
  double dimc, dimrho, diml;
  // 0: reference arithmetic.  1: on the eight strips that the receiver reverses,
  // evaluate the receiver-frame metric at the receiver's (mirrored) edge index.
  int fix_reversed_rotation = 0;
  // source term of the v_r equation (compute_rhs_acoustic.f90:92-116): 0 off, 1 analytic
  // (centre plane f_kcenter instead of the hard-coded gr(200)), 2 sampled S_t at e_rad
  int forcing = 0, f_kcenter = 0, f_nstep = 0, f_nt = 0, e_rad = 0;
  std::vector<double> f_samples;                      // S_t [zone][n][j][i]
  // COMMON /TSTEP/ time, the driver's step, and LAGRANGE_INTERP's saved state
  // (/STEP_TRACK/, /TIME_INTERP/, /LAGRANGE_TIME_INTERP/); advanced by RK4
  mutable double time = 0.0;
  mutable int step = 0, step_old = 0, f_error = 0;
  mutable double xn[7] = {0, 0, 0, 0, 0, 0, 0};
  mutable std::vector<double> LC;                     // [7][zone][j][i]
};

namespace {

inline size_t idx3(const oracle_ctx& c, int k, int j, int i) {
  return (size_t)k * c.plane + (size_t)j * c.nx + i;
}

// ---------------------------------------------------------------- setup
// metric.f90:8-160  SETUP_COORDINATES_METRICS_ALL (xrank = yrank = rrank = 0)
void setup_metric(oracle_ctx& c) {
  const int nx = c.nx, nr = c.nr;
  c.gxi.resize(nx); c.geta.resize(nx); c.gchi.resize(nr);
  for (int i = 1; i <= nx; ++i) {
    double v = -PI * 0.25 + (double(i) - 1.0) * PI * 0.5 / (double(nx) - 1.0);
    c.gxi[i - 1] = v; c.geta[i - 1] = v;
  }
  for (int i = 1; i <= nr; ++i) c.gchi[i - 1] = 0.0 + (double(i) - 1.0) * 1.0 / (double(nr) - 1.0);
  c.dxi = c.gxi[1] - c.gxi[0];
  c.deta = c.dxi;
  c.dchi = c.gchi[1] - c.gchi[0];
  // radial metric dr/dchi by the DRP stencil (metric.f90:48-67)
  c.gdrdchi.assign(nr, 0.0);
  for (int kk = NST + 1; kk <= nr - NST; ++kk) {
    double s = 0.0;
    for (int it = -NST; it <= NST; ++it) s = s + (1.0 / c.dchi) * COEFFS1[it + 3] * c.gr[kk + it - 1];
    c.gdrdchi[kk - 1] = s;
  }
  for (int kk = 1; kk <= NST; ++kk) {
    double s = 0.0;
    for (int it = 1; it <= NSTENCIL; ++it) s = s + (1.0 / c.dchi) * BDY1[kk - 1][it - 1] * c.gr[it - 1];
    c.gdrdchi[kk - 1] = s;
  }
  for (int kk = nr - NST + 1; kk <= nr; ++kk) {
    double s = 0.0;
    for (int it = 1; it <= NSTENCIL; ++it)
      s = s - (1.0 / c.dchi) * BDY1[nr - kk][NSTENCIL - it] * c.gr[nr - NSTENCIL + it - 1];
    c.gdrdchi[kk - 1] = s;
  }
  c.tanxi.resize(nx); c.taneta.resize(nx); c.mC.resize(nx); c.mD.resize(nx);
  for (int i = 0; i < nx; ++i) {
    c.tanxi[i] = std::tan(c.gxi[i]);
    c.taneta[i] = std::tan(c.geta[i]);
    c.mC[i] = std::sqrt(1.0 + c.tanxi[i] * c.tanxi[i]);
    c.mD[i] = std::sqrt(1.0 + c.taneta[i] * c.taneta[i]);
  }
  c.delta.resize(c.plane); c.sdelta.resize(c.plane); c.XY.resize(c.plane); c.CD.resize(c.plane);
  for (int j = 0; j < nx; ++j)
    for (int i = 0; i < nx; ++i) {
      size_t p = (size_t)j * nx + i;
      c.delta[p] = 1.0 + c.tanxi[i] * c.tanxi[i] + c.taneta[j] * c.taneta[j];
      c.sdelta[p] = std::sqrt(1.0 + c.tanxi[i] * c.tanxi[i] + c.taneta[j] * c.taneta[j]);
      c.XY[p] = c.tanxi[i] * c.taneta[j];
      c.CD[p] = c.mC[i] * c.mD[j];
    }
  // interpolation target points (metric.f90:89-91)
  c.interpoints.resize(3 * nx);
  for (int m = 1; m <= 3; ++m)
    for (int t = 0; t < nx; ++t)
      c.interpoints[(m - 1) * nx + t] = std::atan(std::tan(c.geta[t]) / std::tan(c.gxi[nx - 1] + m * c.dxi));
  // spherical coordinates per zone (metric.f90:95-158)
  c.theta.resize(6 * c.plane); c.phi.resize(6 * c.plane);
  for (int z = 1; z <= 6; ++z)
    for (int j = 0; j < nx; ++j)
      for (int i = 0; i < nx; ++i) {
        double ph = 0.0, th = 0.0;
        const double tx = c.tanxi[i], ty = c.taneta[j];
        if (z == 1) {
          ph = c.gxi[i];
          th = std::atan(1.0 / (ty * std::cos(ph)));
          if (th < 0) th += PI;
        } else if (z == 2) {
          ph = c.gxi[i] + PI * 0.5;
          th = std::atan(1.0 / (ty * std::sin(ph)));
          if (th < 0) th += PI;
          if (ph < 0) ph += 2.0 * PI;
        } else if (z == 3) {
          ph = c.gxi[i] + PI;
          th = std::atan(-1.0 / (ty * std::cos(ph)));
          if (th < 0) th += PI;
          if (ph < 0) ph += 2.0 * PI;
        } else if (z == 4) {
          ph = c.gxi[i] + PI * 1.5;
          th = std::atan(-1.0 / (ty * std::sin(ph)));
          if (th < 0) th += PI;
          if (ph < 0) ph += 2.0 * PI;
        } else if (z == 5) {
          th = std::atan(std::sqrt(tx * tx + ty * ty));
          ph = std::atan2(tx, -ty);
          if (ph < 0) ph += 2.0 * PI;
        } else {
          th = PI - std::atan(std::sqrt(tx * tx + ty * ty));
          ph = std::atan2(tx, ty);
          if (ph < 0) ph += 2.0 * PI;
        }
        c.theta[(z - 1) * c.plane + (size_t)j * nx + i] = th;
        c.phi[(z - 1) * c.plane + (size_t)j * nx + i] = ph;
      }
}

// interpolation.f90:9-54  SETUP_LAGRANGE_INTERPOLANT
void setup_lagrange(oracle_ctx& c) {
  const int nx = c.nx;
  c.interpolant.assign(3 * nx * 9, 0.0);
  auto W = [&](int ipoint, int i, int k) -> double& {  // interpolant(ipoint, i, k), 1-based i,k
    return c.interpolant[((size_t)(k - 1) * nx + (i - 1)) * 9 + (ipoint + 4)];
  };
  for (int k = 1; k <= NST; ++k) {
    W(k, 1, k) = 1.0;
    W(-k, nx, k) = 1.0;
    for (int i = 2; i <= nx - 1; ++i) {
      int lower = -NORD, upper = NORD;
      if (i < NORD + 1) lower = -i + 1;
      if (i > nx - NORD) upper = nx - i;
      for (int ip = lower; ip <= upper; ++ip) W(ip, i, k) = 1.0;
      for (int ip = lower; ip <= upper; ++ip)
        for (int it = lower; it <= upper; ++it)
          if (it != ip)
            W(ip, i, k) = (c.interpoints[(k - 1) * nx + (i - 1)] - c.geta[i + it - 1]) * W(ip, i, k) /
                          (c.geta[i + ip - 1] - c.geta[i + it - 1]);
    }
  }
}

// ic_acoustic_wave.f90:61-108  SOLAR_DATA: read the model rows, normalise by row 1
void solar_data(oracle_ctx& c, const double* model) {
  const int nr = c.nr;
  auto data = [&](int k, int col) { return model[(size_t)(k - 1) * 8 + (col - 1)]; };
  c.dimc = data(1, 2);
  c.dimrho = data(1, 3);
  const double rsun = 695.9894e8;
  c.diml = rsun;
  c.gr.resize(nr); c.c2.resize(nr); c.rho0.resize(nr); c.g0.resize(nr);
  for (int k = 1; k <= nr; ++k) {
    c.gr[k - 1] = data(k, 1);
    double cs = data(k, 2) / c.dimc;
    c.c2[k - 1] = std::pow(data(k, 2) / c.dimc, 2.0);
    (void)cs;
    c.rho0[k - 1] = data(k, 3) / c.dimrho;
    c.g0[k - 1] = data(k, 6) * c.diml / std::pow(c.dimc, 2.0);
  }
}

// sponge.f90:18-46 sigma_r(gk); the ratio is a default-REAL (single precision)
// division promoted to double for **s_exp.
void setup_sponge(oracle_ctx& c, double a, double s_exp, int len, int lower, int upper) {
  c.sigma.assign(c.nr, 0.0);
  const int start_lower = len, start_upper = c.nr - len + 1;
  for (int gk = 1; gk <= c.nr; ++gk) {
    double s = 0.0;
    if (upper && gk >= start_upper) {
      float ratio = (float)(gk - start_upper) / (float)len;
      s = a * std::pow((double)ratio, s_exp);
    } else if (lower && gk <= start_lower) {
      float ratio = (float)(start_lower - gk) / (float)len;
      s = a * std::pow((double)ratio, s_exp);
    }
    c.sigma[gk - 1] = s;
  }
}

// ---------------------------------------------------------------- interpolation
// interpolation.f90:261-378 INTERPOLATE_ALONG_X for one layer line (xrank = 0 = px-1):
// in[t] are the source values along the edge, out[t] the interpolated ghost values.
inline void interp_line(const oracle_ctx& c, int layer, const double* in, int stride, double* out) {
  const int mx = c.nx, j = layer;  // j = layer 1..3
  auto W = [&](int it, int ii) { return c.interpolant[((size_t)(j - 1) * mx + (ii - 1)) * 9 + (it + 4)]; };
  auto IN = [&](int i) { return in[(size_t)(i - 1) * stride]; };
  out[0] = IN(j + 1);
  out[mx - 1] = IN(mx - j);
  for (int i = NORD + 1; i <= mx - NORD; ++i) {
    double s = 0.0;
    for (int it = -NORD; it <= NORD; ++it) s = s + IN(i + it) * W(it, i);
    out[i - 1] = s;
  }
  for (int i = 2; i <= NORD; ++i) {
    double s = 0.0;
    for (int it = -i + 1; it <= NORD; ++it) s = s + IN(it + i) * W(it, i);
    out[i - 1] = s;
  }
  for (int i = mx - NORD + 1; i <= mx - 1; ++i) {
    double s = 0.0;
    for (int it = -NORD; it <= mx - i; ++it) s = s + IN(i + it) * W(it, i);
    out[i - 1] = s;
  }
}

// The four edge strips of one zone's field (grad.f90:187-190, filter.f90:25-28):
//  S = INTERPOLATE_ALONG_X(a(:,2:4,:)),  N = INTERPOLATE_ALONG_X(a(:,my-1:my-3:-1,:)),
//  W = INTERPOLATE_ALONG_Y(a(2:4,:,:)),  E = INTERPOLATE_ALONG_Y(a(mx-1:mx-3:-1,:,:)).
// INTERPOLATE_ALONG_Y (interpolation.f90:140-257) is the same line operator along j.
void zone_strips(const oracle_ctx& c, const double* f, double* s /* [4][nr][3][nx] */) {
  const int n = c.nx;
  const size_t ss = (size_t)c.nr * 3 * n;
#pragma omp parallel for schedule(static)
  for (int k = 0; k < c.nr; ++k) {
    const double* fk = f + (size_t)k * c.plane;
    for (int m = 1; m <= 3; ++m) {
      double* oS = s + 0 * ss + ((size_t)k * 3 + (m - 1)) * n;
      double* oN = s + 1 * ss + ((size_t)k * 3 + (m - 1)) * n;
      double* oW = s + 2 * ss + ((size_t)k * 3 + (m - 1)) * n;
      double* oE = s + 3 * ss + ((size_t)k * 3 + (m - 1)) * n;
      interp_line(c, m, fk + (size_t)m * n, 1, oS);               // row j = 1+m
      interp_line(c, m, fk + (size_t)(n - 1 - m) * n, 1, oN);     // row j = my-m
      interp_line(c, m, fk + m, n, oW);                           // column i = 1+m
      interp_line(c, m, fk + (n - 1 - m), n, oE);                 // column i = mx-m
    }
  }
}

// Assemble the (fp, fn) halos of every zone for one direction from all zones' strips.
// halo[zone][side][k][layer][t]
void route_halos(const oracle_ctx& c, const std::vector<double>& strips, const Route (*R)[2],
                 std::vector<double>& halo) {
  const int n = c.nx;
  const size_t ss = (size_t)c.nr * 3 * n;
  halo.resize((size_t)6 * 2 * ss);
  for (int z = 0; z < 6; ++z)
    for (int side = 0; side < 2; ++side) {
      const Route r = R[z][side];
      const double* src = strips.data() + ((size_t)r.src * 4 + r.edge) * ss;
      double* dst = halo.data() + ((size_t)z * 2 + side) * ss;
      for (size_t row = 0; row < (size_t)c.nr * 3; ++row)
        for (int t = 0; t < n; ++t) dst[row * n + t] = src[row * n + (r.rev ? (n - 1 - t) : t)];
    }
}

void all_strips(const oracle_ctx& c, const double* f, std::vector<double>& strips) {
  const size_t ss = (size_t)c.nr * 3 * c.nx;
  strips.resize((size_t)6 * 4 * ss);
  for (int z = 0; z < 6; ++z) zone_strips(c, f + z * c.vol, strips.data() + (size_t)z * 4 * ss);
}

// ---------------------------------------------------------------- derivatives / filters
// Shared body of DDX (derivative.f90:454-599) and FILTER_XI (filter.f90:173-315): a
// centred (2*NST+1)-tap stencil along i with the received halos fp (i = 0,-1,-2) and
// fn (i = mx+1, ...).  fac scales each tap (1/dxi for DDX, 1 for the filter).
void xi_stencil(const oracle_ctx& c, const double* f, const double* fp, const double* fn,
                const double* coef, double fac, double* out) {
  const int mx = c.nx, my = c.nx, mr = c.nr;
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= mr; ++k) {
    const double* fk = f + (size_t)(k - 1) * c.plane;
    double* ok = out + (size_t)(k - 1) * c.plane;
    auto F = [&](int i, int j) { return fk[(size_t)(j - 1) * mx + (i - 1)]; };
    auto FP = [&](int m, int j) { return fp[((size_t)(k - 1) * 3 + (m - 1)) * my + (j - 1)]; };
    auto FN = [&](int m, int j) { return fn[((size_t)(k - 1) * 3 + (m - 1)) * my + (j - 1)]; };
    for (int j = 1; j <= my; ++j) {
      for (int i = NST + 1; i <= mx - NST; ++i) {
        double s = 0.0;
        for (int it = -NST; it <= NST; ++it) s = s + fac * coef[it + 3] * F(i + it, j);
        ok[(size_t)(j - 1) * mx + (i - 1)] = s;
      }
      for (int i = 1; i <= NST; ++i) {
        double s = 0.0;
        for (int it = -NST; it <= -i; ++it) s = s + fac * coef[it + 3] * FP(-i - it + 1, j);
        for (int it = -i + 1; it <= NST; ++it) s = s + fac * coef[it + 3] * F(i + it, j);
        ok[(size_t)(j - 1) * mx + (i - 1)] = s;
      }
      for (int i = mx - NST + 1; i <= mx; ++i) {
        double s = 0.0;
        for (int it = -NST; it <= mx - i; ++it) s = s + fac * coef[it + 3] * F(i + it, j);
        for (int it = mx - i + 1; it <= NST; ++it) s = s + fac * coef[it + 3] * FN(i + it - mx, j);
        ok[(size_t)(j - 1) * mx + (i - 1)] = s;
      }
    }
  }
}

// Shared body of DDY (derivative.f90:135-320) and FILTER_ETA (filter.f90:445-629).
void eta_stencil(const oracle_ctx& c, const double* f, const double* fp, const double* fn,
                 const double* coef, double fac, double* out) {
  const int mx = c.nx, my = c.nx, mr = c.nr;
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= mr; ++k) {
    const double* fk = f + (size_t)(k - 1) * c.plane;
    double* ok = out + (size_t)(k - 1) * c.plane;
    auto F = [&](int i, int j) { return fk[(size_t)(j - 1) * mx + (i - 1)]; };
    auto FP = [&](int i, int m) { return fp[((size_t)(k - 1) * 3 + (m - 1)) * mx + (i - 1)]; };
    auto FN = [&](int i, int m) { return fn[((size_t)(k - 1) * 3 + (m - 1)) * mx + (i - 1)]; };
    for (int j = NST + 1; j <= my - NST; ++j)
      for (int i = 1; i <= mx; ++i) {
        double s = 0.0;
        for (int it = -NST; it <= NST; ++it) s = s + fac * coef[it + 3] * F(i, j + it);
        ok[(size_t)(j - 1) * mx + (i - 1)] = s;
      }
    for (int j = 1; j <= NST; ++j)
      for (int i = 1; i <= mx; ++i) {
        double s = 0.0;
        for (int it = -NST; it <= -j; ++it) s = s + fac * coef[it + 3] * FP(i, -it - j + 1);
        for (int it = -j + 1; it <= NST; ++it) s = s + fac * coef[it + 3] * F(i, it + j);
        ok[(size_t)(j - 1) * mx + (i - 1)] = s;
      }
    for (int j = my - NST + 1; j <= my; ++j)
      for (int i = 1; i <= mx; ++i) {
        double s = 0.0;
        for (int it = -NST; it <= my - j; ++it) s = s + fac * coef[it + 3] * F(i, it + j);
        for (int it = my - j + 1; it <= NST; ++it) s = s + fac * coef[it + 3] * FN(i, it + j - my);
        ok[(size_t)(j - 1) * mx + (i - 1)] = s;
      }
  }
}

// derivative.f90:605-758  DDR with rrank = 0 = pr-1: one-sided Tam-Dong rows at both ends.
void ddr_zone(const oracle_ctx& c, const double* f, double* out) {
  const int mx = c.nx, my = c.nx, mr = c.nr;
  const double fac = 1.0 / c.dchi;
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= mr; ++k) {
    double* ok = out + (size_t)(k - 1) * c.plane;
    for (int p = 0; p < mx * my; ++p) {
      double s = 0.0;
      if (k >= NST + 1 && k <= mr - NST) {
        const double fac2 = fac / c.gdrdchi[k - 1];
        for (int it = -NST; it <= NST; ++it) s = s + fac2 * COEFFS1[it + 3] * f[(size_t)(k + it - 1) * c.plane + p];
      } else if (k <= NST) {
        const double fac2 = fac / c.gdrdchi[k - 1];
        for (int it = 1; it <= NSTENCIL; ++it) s = s + fac2 * BDY1[k - 1][it - 1] * f[(size_t)(it - 1) * c.plane + p];
      } else {
        const double fac2 = -fac / c.gdrdchi[k - 1];
        for (int it = 1; it <= NSTENCIL; ++it)
          s = s + fac2 * BDY1[mr - k][NSTENCIL - it] * f[(size_t)(mr - NSTENCIL + it - 1) * c.plane + p];
      }
      ok[p] = s;
    }
  }
}

// filter.f90:633-781  FILTER_R with rrank = 0 = pr-1: the 5 end planes stay 0 (the
// boundary filter body is commented out at filter.f90:734, 770).
void filter_r_zone(const oracle_ctx& c, const double* g, double* gf) {
  const int mr = c.nr;
#pragma omp parallel for schedule(static)
  for (int k = 1; k <= mr; ++k) {
    double* ok = gf + (size_t)(k - 1) * c.plane;
    if (k >= NSTR + 1 && k <= mr - NSTR) {
      for (size_t p = 0; p < c.plane; ++p) {
        double s = 0.0;
        for (int it = -NSTR; it <= NSTR; ++it) s = s + FILT_R[it + 5] * g[(size_t)(k + it - 1) * c.plane + p];
        ok[p] = s;
      }
    } else {
      for (size_t p = 0; p < c.plane; ++p) ok[p] = 0.0;
    }
  }
}

// ---------------------------------------------------------------- vector transforms
// transform.f90:8-59  CONVERT_XI_ETA_TO_THETA_PHI for zone z (1..6)
void convert_xe_tp(const oracle_ctx& c, int z, const double* axi, const double* aeta, double* ath,
                   double* aph) {
  const int n = c.nx;
#pragma omp parallel for schedule(static)
  for (int k = 0; k < c.nr; ++k)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        const size_t p = (size_t)j * n + i, q = idx3(c, k, j, i);
        if (z <= 4) {
          ath[q] = c.XY[p] / c.CD[p] * axi[q] - aeta[q];
          aph[q] = c.sdelta[p] / c.CD[p] * axi[q];
        } else {
          const double factor = 1.0 / std::sqrt(c.delta[p] - 1.0);
          const double tx = c.tanxi[i], ty = c.taneta[j];
          if (z == 5) {
            ath[q] = factor * (tx / c.mD[j] * axi[q] + ty / c.mC[i] * aeta[q]);
            aph[q] = factor * (-(c.sdelta[p] * ty / c.mD[j] * axi[q]) + c.sdelta[p] * tx / c.mC[i] * aeta[q]);
          } else {
            ath[q] = -(factor * (tx / c.mD[j] * axi[q] + ty / c.mC[i] * aeta[q]));
            aph[q] = factor * (c.sdelta[p] * ty / c.mD[j] * axi[q] - c.sdelta[p] * tx / c.mC[i] * aeta[q]);
          }
        }
      }
}

// transform.f90:114-276  TRANSFORM_VECTOR_BETWEEN_MESHES_DIV for zone z (1..6).  th/ph are
// the zone's interpolated theta/phi strips [edge][k][layer][t]; out receives the
// receiver-frame component strips that this zone sends: E/W -> xi (zones 1-4), and the
// per-zone S/N (or all four for zones 5, 6) strips listed in the reference.
void transform_div(const oracle_ctx& c, int z, const double* th, const double* ph, double* out) {
  const int n = c.nx;
  const size_t ss = (size_t)c.nr * 3 * n;
  double X[7], Y[7], C[7];  // index m+3, m = -3..3
  for (int i = 1; i <= NST; ++i) {
    X[3 - i] = std::tan(c.gxi[0] - i * c.dxi);
    Y[3 - i] = std::tan(c.geta[0] - i * c.deta);
    C[3 - i] = std::sqrt(1.0 + X[3 - i] * X[3 - i]);
    X[3 + i] = std::tan(c.gxi[n - 1] + i * c.dxi);
    Y[3 + i] = std::tan(c.geta[n - 1] + i * c.deta);
    C[3 + i] = std::sqrt(1.0 + X[3 + i] * X[3 + i]);
  }
  std::vector<double> gD(n);
  for (int i = 0; i < n; ++i) gD[i] = std::pow(1.0 + std::pow(std::tan(c.geta[i]), 2.0), 0.5);
  auto S = [&](const double* a, int e, int k, int m, int t) { return a[e * ss + ((size_t)k * 3 + (m - 1)) * n + t]; };
  auto O = [&](int e, int k, int m, int t) -> double& { return out[e * ss + ((size_t)k * 3 + (m - 1)) * n + t]; };
  // The reference evaluates the receiver metric at the sender's own edge index t; the
  // receiver reverses these strips (derivative.f90:217-282, 539-561), so the metric
  // actually belongs at n-1-t.  Only used when fix_reversed_rotation is set.
  auto rev_strip = [&](int e) {
    return (z == 2 && e == ES) || (z == 3 && (e == ES || e == EN)) || (z == 4 && e == EN) ||
           (z == 5 && (e == EN || e == EW)) || (z == 6 && (e == ES || e == EE));
  };
  auto mt = [&](int e, int t) { return (c.fix_reversed_rotation && rev_strip(e)) ? n - 1 - t : t; };
  for (int k = 0; k < c.nr; ++k)
    for (int m = 1; m <= 3; ++m)
      for (int t = 0; t < n; ++t) {
        if (z <= 4) {  // transform.f90:161-179
          const double tg = std::tan(c.geta[t]);
          O(EE, k, m, t) = C[3 - m] * gD[t] / std::sqrt(1.0 + X[3 - m] * X[3 - m] + tg * tg) * S(ph, EE, k, m, t);
          O(EW, k, m, t) = C[3 + m] * gD[t] / std::sqrt(1.0 + X[3 + m] * X[3 + m] + tg * tg) * S(ph, EW, k, m, t);
        }
        if (z == 5 || z == 6) {  // transform.f90:184-221
          const double Ym = (z == 5) ? Y[3 + m] : Y[3 - m];
          for (int e : {ES, EE, EN, EW}) {
            const double tx = std::tan(c.gxi[mt(e, t)]);
            const double f = tx * Ym / std::sqrt(1.0 + tx * tx + Ym * Ym);
            O(e, k, m, t) = -S(th, e, k, m, t) + f * S(ph, e, k, m, t);
          }
        }
        // faces 1-4 onto face 5 (transform.f90:226-248)
        {
          const int tn = mt(EN, t);
          const double tx = std::tan(c.gxi[tn]), ty = std::tan(c.geta[tn]);
          if (z == 1 || z == 3) {
            const double Ym = (z == 1) ? Y[3 - m] : Y[3 + m];
            const double s1 = std::sqrt(tx * tx + Ym * Ym), s2 = std::sqrt(1.0 + tx * tx + Ym * Ym);
            O(EN, k, m, t) = c.mC[tn] * Ym / s1 * S(th, EN, k, m, t) + c.mC[tn] / s1 * tx / s2 * S(ph, EN, k, m, t);
          } else if (z == 2 || z == 4) {
            const double Xm = (z == 2) ? X[3 + m] : X[3 - m];
            const double s1 = std::sqrt(Xm * Xm + ty * ty), s2 = std::sqrt(1.0 + Xm * Xm + ty * ty);
            O(EN, k, m, t) = gD[tn] * Xm / s1 * S(th, EN, k, m, t) - gD[tn] / s1 * ty / s2 * S(ph, EN, k, m, t);
          }
        }
        // faces 1-4 onto face 6 (transform.f90:252-274)
        {
          const int ts = mt(ES, t);
          const double tx = std::tan(c.gxi[ts]), ty = std::tan(c.geta[ts]);
          if (z == 1 || z == 3) {
            const double Ym = (z == 1) ? Y[3 + m] : Y[3 - m];
            const double s1 = std::sqrt(tx * tx + Ym * Ym), s2 = std::sqrt(1.0 + tx * tx + Ym * Ym);
            O(ES, k, m, t) = -(c.mC[ts] * Ym / s1 * S(th, ES, k, m, t)) - c.mC[ts] / s1 * tx / s2 * S(ph, ES, k, m, t);
          } else if (z == 2 || z == 4) {
            const double Xm = (z == 2) ? X[3 + m] : X[3 - m];
            const double s1 = std::sqrt(Xm * Xm + ty * ty), s2 = std::sqrt(1.0 + Xm * Xm + ty * ty);
            O(ES, k, m, t) = -(gD[ts] * Xm / s1 * S(th, ES, k, m, t)) + gD[ts] / s1 * ty / s2 * S(ph, ES, k, m, t);
          }
        }
      }
}

// transform.f90:279-498  TRANSFORM_VECTOR_BETWEEN_MESHES_CURL for zone z (1..6): both
// receiver-frame components (xi, eta) of every strip this zone sends, from its interpolated
// theta/phi strips.  Layout as transform_div: [edge][k][layer][t].
void transform_curl(const oracle_ctx& c, int z, const double* th, const double* ph, double* oxi, double* oeta) {
  const int n = c.nx;
  const size_t ss = (size_t)c.nr * 3 * n;
  double X[7], Y[7], C[7], D[7];  // index m+3, m = -3..3
  for (int i = 1; i <= NST; ++i) {
    X[3 - i] = std::tan(c.gxi[0] - i * c.dxi);
    Y[3 - i] = std::tan(c.geta[0] - i * c.deta);
    C[3 - i] = std::sqrt(1.0 + X[3 - i] * X[3 - i]);
    D[3 - i] = std::sqrt(1.0 + Y[3 - i] * Y[3 - i]);
    X[3 + i] = std::tan(c.gxi[n - 1] + i * c.dxi);
    Y[3 + i] = std::tan(c.geta[n - 1] + i * c.deta);
    C[3 + i] = std::sqrt(1.0 + X[3 + i] * X[3 + i]);
    D[3 + i] = std::sqrt(1.0 + Y[3 + i] * Y[3 + i]);
  }
  std::vector<double> gC(n), gD(n);
  for (int i = 0; i < n; ++i) {
    gC[i] = std::pow(1.0 + std::pow(std::tan(c.gxi[i]), 2.0), 0.5);
    gD[i] = std::pow(1.0 + std::pow(std::tan(c.geta[i]), 2.0), 0.5);
  }
  auto S = [&](const double* a, int e, int k, int m, int t) { return a[e * ss + ((size_t)k * 3 + (m - 1)) * n + t]; };
  auto OX = [&](int e, int k, int m, int t) -> double& { return oxi[e * ss + ((size_t)k * 3 + (m - 1)) * n + t]; };
  auto OE = [&](int e, int k, int m, int t) -> double& { return oeta[e * ss + ((size_t)k * 3 + (m - 1)) * n + t]; };
  // the reversed strips (see transform_div): metric at the receiver's index when fixed
  auto rev_strip = [&](int e) {
    return (z == 2 && e == ES) || (z == 3 && (e == ES || e == EN)) || (z == 4 && e == EN) ||
           (z == 5 && (e == EN || e == EW)) || (z == 6 && (e == ES || e == EE));
  };
  auto mt = [&](int e, int t) { return (c.fix_reversed_rotation && rev_strip(e)) ? n - 1 - t : t; };
  for (int k = 0; k < c.nr; ++k)
    for (int m = 1; m <= 3; ++m)
      for (int t = 0; t < n; ++t) {
        if (z <= 4) {  // transform.f90:314-332
          for (int e : {EE, EW}) {
            const int tj = mt(e, t);
            const double Xm = (e == EE) ? X[3 - m] : X[3 + m], Cm = (e == EE) ? C[3 - m] : C[3 + m];
            const double tg = std::tan(c.geta[tj]);
            OX(e, k, m, t) = Cm * gD[tj] / std::sqrt(1.0 + Xm * Xm + tg * tg) * S(ph, e, k, m, t);
            OE(e, k, m, t) = -S(th, e, k, m, t) + Xm * tg / std::sqrt(1.0 + Xm * Xm + tg * tg) * S(ph, e, k, m, t);
          }
        } else {        // transform.f90:339-390 (faces 5, 6 onto 1-4)
          const double Ym = (z == 5) ? Y[3 + m] : Y[3 - m], Dm = (z == 5) ? D[3 + m] : D[3 - m];
          for (int e : {ES, EN}) {
            const int ti = mt(e, t);
            const double tx = std::tan(c.gxi[ti]);
            OE(e, k, m, t) = -S(th, e, k, m, t) + tx * Ym / std::sqrt(1.0 + tx * tx + Ym * Ym) * S(ph, e, k, m, t);
            OX(e, k, m, t) = c.mC[ti] * Dm / std::sqrt(1.0 + tx * tx + Ym * Ym) * S(ph, e, k, m, t);
          }
          for (int e : {EE, EW}) {
            const int ti = mt(e, t);
            const double tx = std::tan(c.gxi[ti]);
            OE(e, k, m, t) = -S(th, e, k, m, t) + tx * Ym / std::sqrt(1.0 + tx * tx + Ym * Ym) * S(ph, e, k, m, t);
            OX(e, k, m, t) = gC[ti] * Dm / std::sqrt(1.0 + tx * tx + Ym * Ym) * S(ph, e, k, m, t);
          }
        }
        // faces 1-4 onto face 5 (north, transform.f90:396-441) and face 6 (south, :446-493)
        if (z <= 4) {
          for (int e : {EN, ES}) {
            const int ti = mt(e, t);
            const double sg = (e == EN) ? 1.0 : -1.0;
            const double thv = S(th, e, k, m, t), phv = S(ph, e, k, m, t);
            if (z == 1 || z == 3) {
              const bool plus = (z == 3) == (e == EN);     // z=1: N -> Y(-j), S -> Y(j); z=3 mirrored
              const double Ym = plus ? Y[3 + m] : Y[3 - m], Dm = plus ? D[3 + m] : D[3 - m];
              const double tx = std::tan(c.gxi[ti]);
              const double s1 = std::sqrt(tx * tx + Ym * Ym), s2 = std::sqrt(1.0 + tx * tx + Ym * Ym);
              OE(e, k, m, t) = sg * c.mC[ti] * Ym / s1 * thv + sg * c.mC[ti] / s1 * tx / s2 * phv;
              OX(e, k, m, t) = sg * Dm * tx / s1 * thv - sg * Dm / s1 * Ym / s2 * phv;
            } else {
              const double Xm = (z == 2) ? X[3 + m] : X[3 - m], Cm = (z == 2) ? C[3 + m] : C[3 - m];
              const double ty = std::tan(c.geta[ti]);
              const double s1 = std::sqrt(Xm * Xm + ty * ty), s2 = std::sqrt(1.0 + Xm * Xm + ty * ty);
              OX(e, k, m, t) = sg * gD[ti] * Xm / s1 * thv - sg * gD[ti] / s1 * ty / s2 * phv;
              OE(e, k, m, t) = sg * Cm * ty / s1 * thv + sg * Cm / s1 * Xm / s2 * phv;
            }
          }
        }
      }
}

// grad.f90:140-255 COMPUTE_CURL over all zones
void curl_all(const oracle_ctx& c, const double* axi, const double* aeta, const double* ar, double* cxi,
              double* ceta, double* cr) {
  const size_t ss = (size_t)c.nr * 3 * c.nx, V = c.vol;
  std::vector<double> sr, hxr, hyr;
  all_strips(c, ar, sr);
  route_halos(c, sr, ROUTE_X, hxr);
  route_halos(c, sr, ROUTE_Y, hyr);
  std::vector<double> th(V), ph(V), sth(4 * ss), sph(4 * ss);
  std::vector<double> sx((size_t)6 * 4 * ss, 0.0), se((size_t)6 * 4 * ss, 0.0);
  for (int z = 0; z < 6; ++z) {
    convert_xe_tp(c, z + 1, axi + z * V, aeta + z * V, th.data(), ph.data());
    zone_strips(c, th.data(), sth.data());
    zone_strips(c, ph.data(), sph.data());
    transform_curl(c, z + 1, sth.data(), sph.data(), sx.data() + (size_t)z * 4 * ss, se.data() + (size_t)z * 4 * ss);
  }
  std::vector<double> hxx, hyx, hxe, hye;
  route_halos(c, sx, ROUTE_X, hxx);
  route_halos(c, sx, ROUTE_Y, hyx);
  route_halos(c, se, ROUTE_X, hxe);
  route_halos(c, se, ROUTE_Y, hye);
  std::vector<double> d_r_xi(V), d_r_eta(V), d_xi_xi(V), d_eta_eta(V), d_eta_xi(V), d_xi_eta(V), d_xi_r(V), d_eta_r(V);
  const int n = c.nx;
  for (int z = 0; z < 6; ++z) {
    auto hp = [&](const std::vector<double>& h, int side) { return h.data() + ((size_t)z * 2 + side) * ss; };
    xi_stencil(c, ar + z * V, hp(hxr, 0), hp(hxr, 1), COEFFS1, 1.0 / c.dxi, d_r_xi.data());
    eta_stencil(c, ar + z * V, hp(hyr, 0), hp(hyr, 1), COEFFS1, 1.0 / c.deta, d_r_eta.data());
    xi_stencil(c, axi + z * V, hp(hxx, 0), hp(hxx, 1), COEFFS1, 1.0 / c.dxi, d_xi_xi.data());
    eta_stencil(c, aeta + z * V, hp(hye, 0), hp(hye, 1), COEFFS1, 1.0 / c.deta, d_eta_eta.data());
    xi_stencil(c, aeta + z * V, hp(hxe, 0), hp(hxe, 1), COEFFS1, 1.0 / c.dxi, d_eta_xi.data());
    eta_stencil(c, axi + z * V, hp(hyx, 0), hp(hyx, 1), COEFFS1, 1.0 / c.deta, d_xi_eta.data());
    ddr_zone(c, axi + z * V, d_xi_r.data());
    ddr_zone(c, aeta + z * V, d_eta_r.data());
#pragma omp parallel for schedule(static)
    for (int k = 0; k < c.nr; ++k)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          const size_t p = (size_t)j * n + i, l = idx3(c, k, j, i), q = z * V + l;
          const double sd = std::sqrt(c.delta[p]), XY = c.XY[p], CD = c.CD[p], rk = c.gr[k];
          cxi[q] = XY / sd * d_xi_r[l] - CD / sd * d_eta_r[l] +
                   (1.0 / rk) * (XY / sd * axi[q] - CD / sd * aeta[q] + sd / c.mD[j] * d_r_eta[l]);
          ceta[q] = CD / sd * d_xi_r[l] - XY / sd * d_eta_r[l] +
                    (1.0 / rk) * (CD / sd * axi[q] - XY / sd * aeta[q] - sd / c.mC[i] * d_r_xi[l]);
          cr[q] = (sd / rk) * (XY / CD * (d_eta_eta[l] / c.mD[j] - d_xi_xi[l] / c.mC[i]) - d_xi_eta[l] / c.mD[j] +
                               d_eta_xi[l] / c.mC[i]);
        }
  }
}

// ---------------------------------------------------------------- grad / div
// grad.f90:13-59 COMPUTE_GRADIENT over all zones
void gradient_all(const oracle_ctx& c, const double* a, double* gx, double* ge, double* gr) {
  std::vector<double> strips, hx, hy, dx(6 * c.vol), de(6 * c.vol);
  all_strips(c, a, strips);
  route_halos(c, strips, ROUTE_X, hx);
  route_halos(c, strips, ROUTE_Y, hy);
  const size_t ss = (size_t)c.nr * 3 * c.nx;
  for (int z = 0; z < 6; ++z) {
    xi_stencil(c, a + z * c.vol, hx.data() + (z * 2 + 0) * ss, hx.data() + (z * 2 + 1) * ss, COEFFS1, 1.0 / c.dxi, dx.data() + z * c.vol);
    eta_stencil(c, a + z * c.vol, hy.data() + (z * 2 + 0) * ss, hy.data() + (z * 2 + 1) * ss, COEFFS1, 1.0 / c.deta, de.data() + z * c.vol);
    ddr_zone(c, a + z * c.vol, gr + z * c.vol);
  }
  const int n = c.nx;
#pragma omp parallel for collapse(2) schedule(static)
  for (int z = 0; z < 6; ++z)
    for (int k = 0; k < c.nr; ++k)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          const size_t p = (size_t)j * n + i, q = z * c.vol + idx3(c, k, j, i);
          gx[q] = (1.0 / c.gr[k]) * (c.mD[j] * dx[q] + c.XY[p] * de[q] / c.mD[j]);
          ge[q] = (1.0 / c.gr[k]) * (c.mC[i] * de[q] + c.XY[p] * dx[q] / c.mC[i]);
        }
}

// grad.f90:62-136 COMPUTE_DIVERGENCE over all zones
void divergence_all(const oracle_ctx& c, const double* axi, const double* aeta, const double* ar,
                    double* div) {
  const size_t ss = (size_t)c.nr * 3 * c.nx;
  std::vector<double> th(c.vol), ph(c.vol);
  std::vector<double> sth(4 * ss), sph(4 * ss);
  std::vector<double> xs((size_t)6 * 4 * ss, 0.0);  // transformed strips of every zone
  for (int z = 0; z < 6; ++z) {
    convert_xe_tp(c, z + 1, axi + z * c.vol, aeta + z * c.vol, th.data(), ph.data());
    zone_strips(c, th.data(), sth.data());
    zone_strips(c, ph.data(), sph.data());
    transform_div(c, z + 1, sth.data(), sph.data(), xs.data() + (size_t)z * 4 * ss);
  }
  std::vector<double> hx, hy, dx(6 * c.vol), de(6 * c.vol), dr(6 * c.vol);
  route_halos(c, xs, ROUTE_X, hx);
  route_halos(c, xs, ROUTE_Y, hy);
  for (int z = 0; z < 6; ++z) {
    xi_stencil(c, axi + z * c.vol, hx.data() + (z * 2 + 0) * ss, hx.data() + (z * 2 + 1) * ss, COEFFS1, 1.0 / c.dxi, dx.data() + z * c.vol);
    eta_stencil(c, aeta + z * c.vol, hy.data() + (z * 2 + 0) * ss, hy.data() + (z * 2 + 1) * ss, COEFFS1, 1.0 / c.deta, de.data() + z * c.vol);
    ddr_zone(c, ar + z * c.vol, dr.data() + z * c.vol);
  }
  const int n = c.nx;
#pragma omp parallel for collapse(2) schedule(static)
  for (int z = 0; z < 6; ++z)
    for (int k = 0; k < c.nr; ++k)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          const size_t p = (size_t)j * n + i, q = z * c.vol + idx3(c, k, j, i);
          div[q] = (1.0 / c.gr[k]) * (c.delta[p] / c.CD[p] * (dx[q] / c.mC[i] + de[q] / c.mD[j]) -
                                      std::tan(c.gxi[i]) / c.mD[j] * axi[q] -
                                      std::tan(c.geta[j]) / c.mC[i] * aeta[q]) +
                   dr[q] + 2.0 * ar[q] / c.gr[k];
        }
}

// interpolation.f90:385-451  LAGRANGE_INTERP: 7-point Lagrange interpolation in time of the
// sampled source S_t; the nodes and coefficients are refreshed only when floor(xt) advances,
// and the interpolant is evaluated at (step-1)*deltat.  Returns forcing [zone][j][i].
void lagrange_interp(const oracle_ctx& c, std::vector<double>& forcing) {
  const size_t P = c.plane, n6 = 6 * P;
  const double cadforcing = 60.0 * c.dimc / c.diml;   // ic_acoustic_wave.f90:113
  double xt = double(c.step) * c.dt / cadforcing + 1.0;
  const int fl = (int)std::floor(xt);
  if (c.LC.size() != 7 * n6) c.LC.assign(7 * n6, 0.0);
  if (c.step_old < fl) {
    double* x = c.xn;
    x[0] = (xt - 4.0) * cadforcing;
    x[1] = (xt - 3.0) * cadforcing;
    x[2] = (xt - 2.0) * cadforcing;
    x[3] = (xt - 1.0) * cadforcing;
    x[4] = (xt)*cadforcing;
    x[5] = (xt + 1.0) * cadforcing;
    x[6] = (xt + 2.0) * cadforcing;
    std::fill(c.LC.begin(), c.LC.end(), 0.0);
    for (int m = 0; m < 7; ++m) {
      bool on;
      if (m <= 3) on = x[m] >= 0;
      else if (m == 4) on = true;
      else if (m == 5) on = fl < c.f_nstep;
      else on = fl < c.f_nstep - 1;
      if (!on) continue;
      const int smp = fl - 3 + m;                    // S_t(:,:,floor(xt)-3+m), 1-based
      if (smp < 1 || smp > c.f_nt) { c.f_error = 1; continue; }
      double den = 0.0;
      bool first = true;
      for (int j = 0; j < 7; ++j) {
        if (j == m) continue;
        den = first ? (x[m] - x[j]) : den * (x[m] - x[j]);
        first = false;
      }
      for (int z = 0; z < 6; ++z)
        for (size_t p = 0; p < P; ++p)
          c.LC[(size_t)m * n6 + z * P + p] = c.f_samples[((size_t)z * c.f_nt + (smp - 1)) * P + p] / den;
    }
    c.step_old = fl;
  }
  xt = (double(c.step) - 1.0) * c.dt;
  const double* x = c.xn;
  forcing.assign(n6, 0.0);
  for (size_t p = 0; p < n6; ++p) {
    double f = 0.0;
    for (int m = 0; m < 7; ++m) {
      double t = c.LC[(size_t)m * n6 + p];
      for (int j = 0; j < 7; ++j)
        if (j != m) t = t * (xt - x[j]);
      f = (m == 0) ? t : f + t;
    }
    forcing[p] = f;
  }
}

// compute_rhs_acoustic.f90:1-159 COMPUTE_RHS.  The source term :92-104 (analytic) or the
// commented sampled form :107-116 is added when the context enables it; the forcing_rms
// file output :119-125 is not reproduced.
void compute_rhs_all(const oracle_ctx& c, const double* q, double* rhs) {
  const size_t V = c.vol;
  auto Q = [&](int z, int m) { return q + ((size_t)z * 5 + m) * V; };
  auto R = [&](int z, int m) { return rhs + ((size_t)z * 5 + m) * V; };
  // gather the per-field six-zone arrays
  std::vector<double> vxi(6 * V), veta(6 * V), vr(6 * V), p(6 * V), div(6 * V), gx(6 * V), ge(6 * V), grr(6 * V);
  for (int z = 0; z < 6; ++z) {
    std::memcpy(vxi.data() + z * V, Q(z, 1), V * sizeof(double));
    std::memcpy(veta.data() + z * V, Q(z, 2), V * sizeof(double));
    std::memcpy(vr.data() + z * V, Q(z, 3), V * sizeof(double));
    std::memcpy(p.data() + z * V, Q(z, 4), V * sizeof(double));
  }
  divergence_all(c, vxi.data(), veta.data(), vr.data(), div.data());
  gradient_all(c, p.data(), gx.data(), ge.data(), grr.data());
  const int n = c.nx;
#pragma omp parallel for collapse(2) schedule(static)
  for (int z = 0; z < 6; ++z)
    for (int k = 0; k < c.nr; ++k) {
      const double rho0 = c.rho0[k], g0 = c.g0[k], dr0 = c.drho0dr[k];
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          const size_t l = idx3(c, k, j, i), g = z * V + l;
          const double c2 = c.c2_3d.empty() ? c.c2[k] : c.c2_3d[g];
          double r1 = -rho0 * div[g];
          r1 = r1 - Q(z, 3)[l] * dr0;
          R(z, 0)[l] = r1;
          R(z, 1)[l] = -gx[g] / rho0;
          R(z, 2)[l] = -ge[g] / rho0;
          R(z, 3)[l] = -grr[g] / rho0;
          R(z, 3)[l] = R(z, 3)[l] - Q(z, 0)[l] * g0 / rho0;
          double r5 = -c2 * rho0 * div[g];
          r5 = r5 + rho0 * g0 * Q(z, 3)[l];
          R(z, 4)[l] = r5;
        }
    }
  if (c.forcing == 1) {
    const double u = c.time * c.diml / c.dimc - 650.0;
    const double mag = std::exp(-(u * u) / (2.0 * 200.0 * 200.0)) * std::cos(4.0 * PI * u / 700.0);
    const double w = 20.0 * c.dxi, wr = 20.0 * c.dchi;
    for (int z = 0; z < 6; ++z)
      for (int k = 0; k < c.nr; ++k)
        for (int j = 0; j < n; ++j)
          for (int i = 0; i < n; ++i) {
            const size_t p = (size_t)z * c.plane + (size_t)j * n + i;
            const double a = (c.theta[p] - PI / 2.0) / w, b = (c.phi[p] - 0.0) / w;
            const double cc = (c.gr[k] - c.gr[c.f_kcenter]) / wr;
            R(z, 3)[idx3(c, k, j, i)] += mag * std::exp(-(a * a) - b * b - cc * cc);
          }
  } else if (c.forcing == 2) {
    std::vector<double> f;
    lagrange_interp(c, f);
    for (int z = 0; z < 6; ++z)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i)
          R(z, 3)[idx3(c, c.e_rad, j, i)] += f[(size_t)z * c.plane + (size_t)j * n + i];
  }
}

// bc_acoustic_wave.f90:1-36  BC_RHS: zero RHS at global k = 1 and k = nr
void bc_rhs_all(const oracle_ctx& c, double* rhs) {
  for (int z = 0; z < 6; ++z)
    for (int m = 0; m < 5; ++m) {
      double* r = rhs + ((size_t)z * 5 + m) * c.vol;
      std::fill(r, r + c.plane, 0.0);
      std::fill(r + (size_t)(c.nr - 1) * c.plane, r + c.vol, 0.0);
    }
}

// sponge.f90:1-58  SPONGE: rhs -= sigma_r (q - 0) for rho, v_r, p
void sponge_all(const oracle_ctx& c, const double* q, double* rhs) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int z = 0; z < 6; ++z)
    for (int k = 0; k < c.nr; ++k) {
      const double s = c.sigma[k];
      for (int m : {0, 3, 4}) {
        const double* qq = q + ((size_t)z * 5 + m) * c.vol + (size_t)k * c.plane;
        double* rr = rhs + ((size_t)z * 5 + m) * c.vol + (size_t)k * c.plane;
        for (size_t p = 0; p < c.plane; ++p) rr[p] = rr[p] - s * (qq[p] - 0.0);
      }
    }
}

// filter.f90:9-48  FILTER_EXP: per field, halos from the unfiltered q, then XI, ETA, R.
void filter_exp_all(const oracle_ctx& c, const double* q, double* qf) {
  const size_t V = c.vol, ss = (size_t)c.nr * 3 * c.nx;
  std::vector<double> f(6 * V), t1(6 * V), t2(6 * V), strips, hx, hy;
  for (int m = 0; m < 5; ++m) {
    for (int z = 0; z < 6; ++z) std::memcpy(f.data() + z * V, q + ((size_t)z * 5 + m) * V, V * sizeof(double));
    all_strips(c, f.data(), strips);
    route_halos(c, strips, ROUTE_X, hx);
    route_halos(c, strips, ROUTE_Y, hy);
    for (int z = 0; z < 6; ++z) {
      xi_stencil(c, f.data() + z * V, hx.data() + (z * 2 + 0) * ss, hx.data() + (z * 2 + 1) * ss, FILT, 1.0, t1.data() + z * V);
      eta_stencil(c, t1.data() + z * V, hy.data() + (z * 2 + 0) * ss, hy.data() + (z * 2 + 1) * ss, FILT, 1.0, t2.data() + z * V);
      filter_r_zone(c, t2.data() + z * V, qf + ((size_t)z * 5 + m) * V);
    }
  }
}

}  // namespace

// ================================================================== C API
extern "C" {

oracle_ctx* oracle_create(int nx, int nr, const double* model, double dt, double a_sponge,
                          double s_exp, int k_sponge_length, int sponge_lower, int sponge_upper,
                          const double* c2_3d) {
  if (nx < 10 || nr < 12 || !model) return nullptr;
  oracle_ctx* c = new oracle_ctx();
  c->nx = nx; c->nr = nr;
  c->plane = (size_t)nx * nx;
  c->vol = c->plane * nr;
  c->dt = dt;
  solar_data(*c, model);
  setup_metric(*c);
  setup_lagrange(*c);
  setup_sponge(*c, a_sponge, s_exp, k_sponge_length, sponge_lower, sponge_upper);
  // DDR(rho0) (compute_rhs_acoustic.f90:51) is a constant of the background: evaluate it
  // once with the same one-sided/centred rows as DDR.
  c->drho0dr.assign(nr, 0.0);
  {
    const double fac = 1.0 / c->dchi;
    for (int k = 1; k <= nr; ++k) {
      double s = 0.0;
      if (k >= NST + 1 && k <= nr - NST) {
        const double fac2 = fac / c->gdrdchi[k - 1];
        for (int it = -NST; it <= NST; ++it) s = s + fac2 * COEFFS1[it + 3] * c->rho0[k + it - 1];
      } else if (k <= NST) {
        const double fac2 = fac / c->gdrdchi[k - 1];
        for (int it = 1; it <= NSTENCIL; ++it) s = s + fac2 * BDY1[k - 1][it - 1] * c->rho0[it - 1];
      } else {
        const double fac2 = -fac / c->gdrdchi[k - 1];
        for (int it = 1; it <= NSTENCIL; ++it) s = s + fac2 * BDY1[nr - k][NSTENCIL - it] * c->rho0[nr - NSTENCIL + it - 1];
      }
      c->drho0dr[k - 1] = s;
    }
  }
  if (c2_3d) c->c2_3d.assign(c2_3d, c2_3d + 6 * c->vol);
  return c;
}

void oracle_destroy(oracle_ctx* c) { delete c; }

void oracle_set_fix_reversed_rotation(oracle_ctx* c, int on) { c->fix_reversed_rotation = on ? 1 : 0; }

void oracle_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int oracle_get_grid(const oracle_ctx* c, int which, double* out) {
  const std::vector<double>* v = nullptr;
  switch (which) {
    case 0: v = &c->theta; break;
    case 1: v = &c->phi; break;
    case 2: v = &c->gxi; break;
    case 3: v = &c->gr; break;
    case 4: v = &c->gdrdchi; break;
    case 5: v = &c->interpolant; break;
    case 6: v = &c->interpoints; break;
    case 7: v = &c->c2; break;
    case 8: v = &c->rho0; break;
    case 9: v = &c->g0; break;
    case 10: v = &c->sigma; break;
    case 11: v = &c->drho0dr; break;
    default: return -1;
  }
  std::memcpy(out, v->data(), v->size() * sizeof(double));
  return (int)v->size();
}

void oracle_add_gaussian(const oracle_ctx* c, double* q, double x0, double y0, double z0, double width,
                         double amp) {
  const int n = c->nx;
#pragma omp parallel for collapse(2) schedule(static)
  for (int z = 0; z < 6; ++z)
    for (int k = 0; k < c->nr; ++k)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          const size_t p = (size_t)z * c->plane + (size_t)j * n + i;
          const double th = c->theta[p], ph = c->phi[p], r = c->gr[k];
          const double x = r * std::sin(th) * std::cos(ph), y = r * std::sin(th) * std::sin(ph),
                       zz = r * std::cos(th);
          const double d2 = (x - x0) * (x - x0) + (y - y0) * (y - y0) + (zz - z0) * (zz - z0);
          q[((size_t)z * 5 + 4) * c->vol + idx3(*c, k, j, i)] += amp * std::exp(-d2 / (2.0 * width * width));
        }
}

void oracle_interpolate_strips(const oracle_ctx* c, const double* f, double* strips) {
  const size_t ss = (size_t)c->nr * 3 * c->nx;
  for (int z = 0; z < 6; ++z) zone_strips(*c, f + z * c->vol, strips + (size_t)z * 4 * ss);
}

void oracle_ddx(const oracle_ctx* c, const double* f, double* out) {
  std::vector<double> strips, hx;
  all_strips(*c, f, strips);
  route_halos(*c, strips, ROUTE_X, hx);
  const size_t ss = (size_t)c->nr * 3 * c->nx;
  for (int z = 0; z < 6; ++z)
    xi_stencil(*c, f + z * c->vol, hx.data() + (z * 2) * ss, hx.data() + (z * 2 + 1) * ss, COEFFS1, 1.0 / c->dxi, out + z * c->vol);
}

void oracle_ddy(const oracle_ctx* c, const double* f, double* out) {
  std::vector<double> strips, hy;
  all_strips(*c, f, strips);
  route_halos(*c, strips, ROUTE_Y, hy);
  const size_t ss = (size_t)c->nr * 3 * c->nx;
  for (int z = 0; z < 6; ++z)
    eta_stencil(*c, f + z * c->vol, hy.data() + (z * 2) * ss, hy.data() + (z * 2 + 1) * ss, COEFFS1, 1.0 / c->deta, out + z * c->vol);
}

void oracle_ddr(const oracle_ctx* c, const double* f, double* out) {
  for (int z = 0; z < 6; ++z) ddr_zone(*c, f + z * c->vol, out + z * c->vol);
}

void oracle_gradient(const oracle_ctx* c, const double* p, double* gxi, double* geta, double* gr) {
  gradient_all(*c, p, gxi, geta, gr);
}

void oracle_divergence(const oracle_ctx* c, const double* vxi, const double* veta, const double* vr,
                       double* div) {
  divergence_all(*c, vxi, veta, vr, div);
}

void oracle_curl(const oracle_ctx* c, const double* axi, const double* aeta, const double* ar, double* cxi,
                 double* ceta, double* cr) {
  curl_all(*c, axi, aeta, ar, cxi, ceta, cr);
}

void oracle_filter_field(const oracle_ctx* c, const double* f, double* out, int which) {
  const size_t ss = (size_t)c->nr * 3 * c->nx;
  std::vector<double> strips, h;
  if (which == 2) {
    for (int z = 0; z < 6; ++z) filter_r_zone(*c, f + z * c->vol, out + z * c->vol);
    return;
  }
  all_strips(*c, f, strips);
  route_halos(*c, strips, which == 0 ? ROUTE_X : ROUTE_Y, h);
  for (int z = 0; z < 6; ++z) {
    if (which == 0)
      xi_stencil(*c, f + z * c->vol, h.data() + (z * 2) * ss, h.data() + (z * 2 + 1) * ss, FILT, 1.0, out + z * c->vol);
    else
      eta_stencil(*c, f + z * c->vol, h.data() + (z * 2) * ss, h.data() + (z * 2 + 1) * ss, FILT, 1.0, out + z * c->vol);
  }
}

void oracle_compute_rhs(const oracle_ctx* c, const double* q, double* rhs) { compute_rhs_all(*c, q, rhs); }
void oracle_bc_rhs(const oracle_ctx* c, double* rhs) { bc_rhs_all(*c, rhs); }
void oracle_sponge(const oracle_ctx* c, const double* q, double* rhs) { sponge_all(*c, q, rhs); }
void oracle_filter_exp(const oracle_ctx* c, const double* q, double* qf) { filter_exp_all(*c, q, qf); }

// timestep.f90:41-86  RK4: five 2N-storage stages, then FILTER_EXP every step.
void oracle_rk4(const oracle_ctx* c, double* q, int nsteps) {
  const size_t N = (size_t)6 * 5 * c->vol;
  std::vector<double> qw(N), rhs(N), qf(N);
  for (int step = 0; step < nsteps; ++step) {
    std::fill(qw.begin(), qw.end(), 0.0);
    for (int k = 0; k < 5; ++k) {
      compute_rhs_all(*c, q, rhs.data());
      bc_rhs_all(*c, rhs.data());
      sponge_all(*c, q, rhs.data());
      const double a = ALPHA_RK4[k], b = BETA_RK4[k], dt = c->dt;
#pragma omp parallel for schedule(static)
      for (long long l = 0; l < (long long)N; ++l) {
        qw[l] = a * qw[l] + dt * rhs[l];
        q[l] = q[l] + b * qw[l];
      }
    }
    filter_exp_all(*c, q, qf.data());
    std::memcpy(q, qf.data(), N * sizeof(double));
    c->time = c->time + c->dt;                         // timestep.f90:82
    c->step = c->step + 1;                             // cube.f90:71 loop counter
  }
}

// Source term selection and its data (see oracle_ctx).
int oracle_set_forcing(oracle_ctx* c, int kind, int k_center, int nstep) {
  if (kind < 0 || kind > 2 || (kind == 1 && (k_center < 0 || k_center >= c->nr))) return -1;
  if (kind == 2 && c->f_samples.empty()) return -1;
  c->forcing = kind;
  c->f_kcenter = k_center;
  c->f_nstep = nstep;
  // e_rad: plane nearest 1 - 100 km / R_sun (ic_acoustic_wave.f90:111, 117-122)
  const double excitdep = 1.0 - 100e5 / c->diml;
  double temp = 1.0;
  for (int k = 0; k < c->nr; ++k)
    if (std::fabs(c->gr[k] - excitdep) <= temp) {
      temp = std::fabs(c->gr[k] - excitdep);
      c->e_rad = k;
    }
  return 0;
}

// READ_FORCING_FUNC (output.f90:271-307): f(i, j, n) stored with n fastest, then j, then i.
int oracle_set_forcing_samples(oracle_ctx* c, int zone, const double* f, int nt) {
  if (zone < 0 || zone > 5 || nt < 1 || (c->f_nt && nt != c->f_nt)) return -1;
  const int n = c->nx;
  if (c->f_samples.empty()) { c->f_samples.assign((size_t)6 * nt * c->plane, 0.0); c->f_nt = nt; }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j)
      for (int m = 0; m < nt; ++m)
        c->f_samples[((size_t)zone * nt + m) * c->plane + (size_t)j * n + i] = f[((size_t)i * n + j) * nt + m];
  return 0;
}

void oracle_set_clock(oracle_ctx* c, double time, int step) {
  c->time = time;
  c->step = step;
  c->step_old = 0;
  for (double& v : c->xn) v = 0.0;
  c->LC.clear();
}

void oracle_get_clock(const oracle_ctx* c, double* time, int* step) {
  if (time) *time = c->time;
  if (step) *step = c->step;
}

// auxiliary.f90:100-125  norm: (sum/(nx*ny*nr)*6)**0.5 over all zones (the reference
// multiplies by 6 where a mean over six zones would divide).
double oracle_norm(const oracle_ctx* c, const double* q, int field) {
  double summ = 0.0;
  for (int z = 0; z < 6; ++z) {
    const double* f = q + ((size_t)z * 5 + (field - 1)) * c->vol;
    for (size_t l = 0; l < c->vol; ++l) summ = summ + std::pow(f[l], 2.0);
  }
  return std::pow(summ / (double(c->nx) * double(c->nx) * double(c->nr)) * 6.0, 0.5);
}

}  // extern "C"
