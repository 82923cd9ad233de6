// tables.cpp -- host-side FP64 setup (product code).  See tables.h.
#include "tables.h"

#include <cmath>
#include <cstdio>

namespace solar {

// Antisymmetric DRP weights c1..c3 (c0 = 0); header:40-46.
const double kDrp[4] = {0.0, 0.79926643, -0.18941314, 0.02651995};
// One-sided rows bdy(row, 1..7); header:49-55 (the DATA statement fills the (3,7) array
// column by column, so row r is every third value starting at r).
const double kBdy[3][7] = {
    {-2.192280339, 4.748611401, -5.108851915, 4.461567104, -2.833498741, 1.128328861, -0.203876371},
    {-0.209337622, -1.084875676, 2.147776050, -1.388928322, 0.768949766, -0.28181465, 0.048230454},
    {0.049041958, -0.468840357, -0.474760914, 1.273274737, -0.518484526, 0.166138533, -0.026369431}};
// header:68-76
const double kAlpha[5] = {0.0, -4.801594388477952e-01, -1.404247195200064e+00,
                          -2.016477077503357e+00, -1.056444269767207e+00};
const double kBeta[5] = {1.028639988104959e-01, 7.408540575766301e-01, 7.426530946683799e-01,
                         4.694937902357905e-01, 1.881733382887932e-01};

// Receiver-centric edge table of the six faces.  It is the message routing of the
// reference's inter-zone halo exchange with one rank per zone: xi-direction halos
// (DDX, derivative.f90:374-452, reversal :539-561; FILTER_XI filter.f90:93-171) fill the
// W (fp) and E (fn) sides, eta-direction halos (DDY, derivative.f90:55-133, reversal
// :217-282; FILTER_ETA filter.f90:364-443) the S (fp) and N (fn) sides.
const EdgeRoute kRoutes[6][4] = {
    // S                N               W               E
    {{5, kN, 0}, {4, kS, 0}, {3, kE, 0}, {1, kW, 0}},   // face 1
    {{5, kE, 1}, {4, kE, 0}, {0, kE, 0}, {2, kW, 0}},   // face 2
    {{5, kS, 1}, {4, kN, 1}, {1, kE, 0}, {3, kW, 0}},   // face 3
    {{5, kW, 0}, {4, kW, 1}, {2, kE, 0}, {0, kW, 0}},   // face 4
    {{0, kN, 0}, {2, kN, 1}, {3, kN, 1}, {1, kN, 0}},   // face 5 (north)
    {{2, kS, 1}, {0, kS, 0}, {3, kS, 0}, {1, kS, 1}},   // face 6 (south)
};

namespace {

// d/dchi of a radial profile with the derivative stencil, one-sided at both ends
// (derivative.f90:656-754 with rrank = 0 = pr - 1; metric.f90:48-67).
std::vector<double> radial_derivative(const std::vector<double>& f, double dchi) {
  const int nr = (int)f.size();
  std::vector<double> d(nr, 0.0);
  for (int k = 0; k < nr; ++k) {
    double s = 0.0;
    if (k >= 3 && k <= nr - 4) {
      for (int m = 1; m <= 3; ++m) s += kDrp[m] * (f[k + m] - f[k - m]);
    } else if (k < 3) {
      for (int m = 0; m < 7; ++m) s += kBdy[k][m] * f[m];
    } else {
      const int row = nr - 1 - k;
      for (int m = 0; m < 7; ++m) s -= kBdy[row][6 - m] * f[nr - 7 + m];
    }
    d[k] = s / dchi;
  }
  return d;
}

}  // namespace

int build_tables(const solar_desc& d, HostTables& t, std::string& err) {
  const int n = d.nx, nr = d.nr;
  if (n < 16 || n % 16 != 0) { err = "nx must be a multiple of 16 and >= 16"; return SOLAR_ERR_ARG; }
  if (nr < 16) { err = "nr must be >= 16"; return SOLAR_ERR_ARG; }
  if (!d.model) { err = "model (solar_model rows) is required"; return SOLAR_ERR_ARG; }
  if (d.sponge_len < 1) { err = "sponge_len must be >= 1"; return SOLAR_ERR_ARG; }
  t.n = n; t.nr = nr;
  const double pi = std::acos(-1.0);

  // SOLAR_DATA (ic_acoustic_wave.f90:73-108): normalise by the first row.
  const double* M = d.model;
  const double dimc = M[1], dimrho = M[2], diml = 695.9894e8;
  t.dimc = dimc;
  if (dimc == 0.0 || dimrho == 0.0) { err = "model row 1 has zero c or rho"; return SOLAR_ERR_ARG; }
  t.gr.resize(nr); t.c2.resize(nr); t.rho0.resize(nr); t.g0.resize(nr);
  for (int k = 0; k < nr; ++k) {
    const double* row = M + (size_t)k * 8;
    t.gr[k] = row[0];
    const double cs = row[1] / dimc;
    t.c2[k] = cs * cs;
    t.rho0[k] = row[2] / dimrho;
    t.g0[k] = row[5] * diml / (dimc * dimc);
    if (!(t.gr[k] > 0.0) || !(t.rho0[k] > 0.0)) { err = "model needs r > 0 and rho > 0"; return SOLAR_ERR_ARG; }
  }

  // Grids (metric.f90:14-45).
  t.gxi.resize(n); t.tanx.resize(n);
  for (int i = 0; i < n; ++i) {
    t.gxi[i] = -pi * 0.25 + double(i) * pi * 0.5 / double(n - 1);
    t.tanx[i] = std::tan(t.gxi[i]);
  }
  t.dxi = t.gxi[1] - t.gxi[0];
  t.dchi = 1.0 / double(nr - 1);
  t.gdrdchi = radial_derivative(t.gr, t.dchi);
  for (int k = 0; k < nr; ++k)
    if (!(t.gdrdchi[k] > 0.0)) { err = "radius must increase with k"; return SOLAR_ERR_ARG; }

  // Radial rows.
  std::vector<double> drho0 = radial_derivative(t.rho0, t.dchi);
  t.radial.assign((size_t)kNumRadial * nr, 0.0);
  auto R = [&](int row, int k) -> double& { return t.radial[(size_t)row * nr + k]; };
  const int start_lower = d.sponge_len, start_upper = nr - d.sponge_len + 1;
  for (int k = 0; k < nr; ++k) {
    const int gk = k + 1;
    R(kInvR, k) = 1.0 / t.gr[k];
    R(kFacR, k) = (1.0 / t.dchi) / t.gdrdchi[k];
    R(kRho0, k) = t.rho0[k];
    R(kInvRho0, k) = 1.0 / t.rho0[k];
    R(kC2Rho0, k) = t.c2[k] * t.rho0[k];
    R(kDRho0, k) = drho0[k] / t.gdrdchi[k];
    R(kG0Rho0, k) = t.g0[k] / t.rho0[k];
    R(kRho0G0, k) = t.rho0[k] * t.g0[k];
    // sponge.f90:40-46; the ratio is a single-precision division in the reference.
    double s = 0.0;
    if (d.sponge_upper && gk >= start_upper) {
      const float ratio = (float)(gk - start_upper) / (float)d.sponge_len;
      s = d.sponge_amp * std::pow((double)ratio, d.sponge_exp);
    } else if (d.sponge_lower && gk <= start_lower) {
      const float ratio = (float)(start_lower - gk) / (float)d.sponge_len;
      s = d.sponge_amp * std::pow((double)ratio, d.sponge_exp);
    }
    R(kSigma, k) = s;
  }
  t.dr_weight.resize(nr);
  for (int k = 0; k < nr; ++k) t.dr_weight[k] = t.gr[k] * t.gr[k] * t.gdrdchi[k] * t.dchi;

  // Horizontal metric (metric.f90:73-85, grad.f90:211-212, 287-289).
  const size_t P2 = (size_t)n * n;
  t.metric.assign((size_t)kNumMetric * P2, 0.0);
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      const double X = t.tanx[i], Y = t.tanx[j];
      const double C = std::sqrt(1.0 + X * X), D = std::sqrt(1.0 + Y * Y);
      const double delta = 1.0 + X * X + Y * Y;
      const size_t p = (size_t)j * n + i;
      t.metric[kMD * P2 + p] = D;
      t.metric[kMXYD * P2 + p] = X * Y / D;
      t.metric[kMC * P2 + p] = C;
      t.metric[kMXYC * P2 + p] = X * Y / C;
      t.metric[kMDivX * P2 + p] = delta / (C * D) / C;
      t.metric[kMDivY * P2 + p] = delta / (C * D) / D;
      t.metric[kMTX * P2 + p] = X / D;
      t.metric[kMTY * P2 + p] = Y / C;
      t.metric[kMVol * P2 + p] = (C * C * D * D) / (delta * std::sqrt(delta)) * t.dxi * t.dxi;
    }

  // Local (v_xi, v_eta) -> global (v_theta, v_phi) of the three face kinds
  // (CONVERT_XI_ETA_TO_THETA_PHI, transform.f90:19-56): theta = a0 v_xi + a1 v_eta,
  // phi = a2 v_xi + a3 v_eta.  Kind 0: faces 1-4, kind 1: face 5, kind 2: face 6.
  t.conv.assign((size_t)3 * 4 * P2, 0.0);
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      const double X = t.tanx[i], Y = t.tanx[j];
      const double C = std::sqrt(1.0 + X * X), D = std::sqrt(1.0 + Y * Y);
      const double delta = 1.0 + X * X + Y * Y, sd = std::sqrt(delta);
      const double f = 1.0 / std::sqrt(delta - 1.0);
      const size_t p = (size_t)j * n + i;
      double a[3][4] = {{X * Y / (C * D), -1.0, sd / (C * D), 0.0},
                        {f * X / D, f * Y / C, -f * sd * Y / D, f * sd * X / C},
                        {-f * X / D, -f * Y / C, f * sd * Y / D, -f * sd * X / C}};
      for (int kind = 0; kind < 3; ++kind)
        for (int e = 0; e < 4; ++e) t.conv[((size_t)kind * 4 + e) * P2 + p] = a[kind][e];
    }

  // Lagrange edge interpolation (metric.f90:89-91, interpolation.f90:22-52).
  std::vector<double> ip(3 * (size_t)n);
  for (int m = 1; m <= 3; ++m)
    for (int q = 0; q < n; ++q)
      ip[(m - 1) * n + q] = std::atan(std::tan(t.gxi[q]) / std::tan(t.gxi[n - 1] + m * t.dxi));
  t.interpolant.assign((size_t)3 * n * 9, 0.0);
  auto W = [&](int layer, int q, int it) -> double& { return t.interpolant[((size_t)layer * n + q) * 9 + it + 4]; };
  for (int m = 1; m <= 3; ++m) {
    W(m - 1, 0, m) = 1.0;
    W(m - 1, n - 1, -m) = 1.0;
    for (int q = 1; q <= n - 2; ++q) {
      int lo = -4, hi = 4;
      if (q < 4) lo = -q;
      if (q > n - 5) hi = n - 1 - q;
      for (int a = lo; a <= hi; ++a) {
        double w = 1.0;
        for (int b = lo; b <= hi; ++b)
          if (b != a) w = (ip[(m - 1) * n + q] - t.gxi[q + b]) * w / (t.gxi[q + a] - t.gxi[q + b]);
        W(m - 1, q, a) = w;
      }
    }
  }
  // Fixed 9-point windows [s0, s0+9) inside the edge; taps outside the reference's
  // shortened stencil get weight 0.
  t.w9.assign((size_t)3 * n * 9, 0.0);
  t.s0.assign((size_t)3 * n, 0);
  for (int l = 0; l < 3; ++l)
    for (int q = 0; q < n; ++q) {
      int s0 = q - 4;
      if (s0 < 0) s0 = 0;
      if (s0 > n - 9) s0 = n - 9;
      t.s0[(size_t)l * n + q] = s0;
      for (int s = 0; s < 9; ++s) {
        const int it = s0 + s - q;
        if (it >= -4 && it <= 4) t.w9[((size_t)l * n + q) * 9 + s] = W(l, q, it);
      }
    }

  // Receiver-frame rotation of the vector strips (TRANSFORM_VECTOR_BETWEEN_MESHES_DIV,
  // transform.f90:142-274), indexed by the SENDING face and edge: ghost value =
  // c_theta * theta_interp + c_phi * phi_interp.  X(+-m), Y(+-m) are the tangents of
  // the receiver's ghost coordinates (transform.f90:142-152).
  double Xp[4], Xm[4];  // X(+m), X(-m), m = 1..3 (Y is identical: geta == gxi)
  for (int m = 1; m <= 3; ++m) {
    Xp[m] = std::tan(t.gxi[n - 1] + m * t.dxi);
    Xm[m] = std::tan(t.gxi[0] - m * t.dxi);
  }
  t.rot.assign((size_t)6 * 4 * 3 * n * 2, 0.0);
  auto ROT = [&](int z, int e, int l, int q, int c) -> double& {
    return t.rot[((((size_t)z * 4 + e) * 3 + l) * n + q) * 2 + c];
  };
  auto reversed_on_receipt = [&](int z, int e) {
    for (int f = 0; f < 6; ++f)
      for (int g = 0; g < 4; ++g)
        if (kRoutes[f][g].src_face == z && kRoutes[f][g].src_edge == e) return kRoutes[f][g].reversed != 0;
    return false;
  };
  for (int z = 0; z < 6; ++z)
    for (int e = 0; e < 4; ++e) {
      const bool mirror = d.fix_reversed_rotation && reversed_on_receipt(z, e);
      for (int l = 0; l < 3; ++l) {
        const int m = l + 1;
        for (int q = 0; q < n; ++q) {
          const int qq = mirror ? n - 1 - q : q;   // receiver's edge index
          const double tq = t.tanx[qq];
          const double Cq = std::sqrt(1.0 + tq * tq);
          double cth = 0.0, cph = 0.0;
          if (z <= 3 && (e == kE || e == kW)) {           // transform.f90:161-179
            const double X = (e == kE) ? Xm[m] : Xp[m];
            cph = std::sqrt(1.0 + X * X) * Cq / std::sqrt(1.0 + X * X + tq * tq);
          } else if (z >= 4) {                             // transform.f90:184-221
            const double Y = (z == 4) ? Xp[m] : Xm[m];
            cth = -1.0;
            cph = tq * Y / std::sqrt(1.0 + tq * tq + Y * Y);
          } else if (z == 0 || z == 2) {                   // faces 1, 3 -> 5 / 6 (eta)
            double Y;
            if (e == kN) Y = (z == 0) ? Xm[m] : Xp[m];
            else Y = (z == 0) ? Xp[m] : Xm[m];
            const double s1 = std::sqrt(tq * tq + Y * Y), s2 = std::sqrt(1.0 + tq * tq + Y * Y);
            const double sg = (e == kN) ? 1.0 : -1.0;
            cth = sg * Cq * Y / s1;
            cph = sg * Cq / s1 * tq / s2;
          } else {                                         // faces 2, 4 -> 5 / 6 (xi)
            const double X = (z == 1) ? Xp[m] : Xm[m];
            const double s1 = std::sqrt(X * X + tq * tq), s2 = std::sqrt(1.0 + X * X + tq * tq);
            const double sg = (e == kN) ? 1.0 : -1.0;
            cth = sg * Cq * X / s1;
            cph = -sg * Cq / s1 * tq / s2;
          }
          ROT(z, e, l, q, 0) = cth;
          ROT(z, e, l, q, 1) = cph;
        }
      }
    }

  // Both receiver-frame components of every vector strip, for COMPUTE_CURL
  // (TRANSFORM_VECTOR_BETWEEN_MESHES_CURL, transform.f90:279-498), indexed like ROT:
  // component out (0 xi, 1 eta) = cth * theta_interp + cph * phi_interp.
  std::vector<double> rotc((size_t)6 * 4 * 3 * n * 4, 0.0);
  auto RC = [&](int z, int e, int l, int q, int o, int c) -> double& {
    return rotc[(((((size_t)z * 4 + e) * 3 + l) * n + q) * 2 + o) * 2 + c];
  };
  for (int z = 0; z < 6; ++z)
    for (int e = 0; e < 4; ++e) {
      const bool mirror = d.fix_reversed_rotation && reversed_on_receipt(z, e);
      for (int l = 0; l < 3; ++l) {
        const int m = l + 1;
        for (int q = 0; q < n; ++q) {
          const int qq = mirror ? n - 1 - q : q;
          const double tq = t.tanx[qq], Cq = std::sqrt(1.0 + tq * tq);
          double xt = 0, xp = 0, et = 0, ep = 0;          // (xi, eta) x (theta, phi)
          if (z <= 3 && (e == kE || e == kW)) {           // transform.f90:314-332
            const double X = (e == kE) ? Xm[m] : Xp[m], sx = std::sqrt(1.0 + X * X + tq * tq);
            xp = std::sqrt(1.0 + X * X) * Cq / sx;
            et = -1.0;
            ep = X * tq / sx;
          } else if (z >= 4) {                             // transform.f90:339-390
            const double Y = (z == 4) ? Xp[m] : Xm[m], sy = std::sqrt(1.0 + tq * tq + Y * Y);
            et = -1.0;
            ep = tq * Y / sy;
            xp = Cq * std::sqrt(1.0 + Y * Y) / sy;
          } else {                                         // faces 1-4 onto 5 / 6 (:396-493)
            const double sg = (e == kN) ? 1.0 : -1.0;
            if (z == 0 || z == 2) {
              const double Y = ((z == 2) == (e == kN)) ? Xp[m] : Xm[m];
              const double s1 = std::sqrt(tq * tq + Y * Y), s2 = std::sqrt(1.0 + tq * tq + Y * Y);
              const double Dy = std::sqrt(1.0 + Y * Y);
              et = sg * Cq * Y / s1;
              ep = sg * Cq / s1 * tq / s2;
              xt = sg * Dy * tq / s1;
              xp = -sg * Dy / s1 * Y / s2;
            } else {
              const double X = (z == 1) ? Xp[m] : Xm[m];
              const double s1 = std::sqrt(X * X + tq * tq), s2 = std::sqrt(1.0 + X * X + tq * tq);
              const double Cx = std::sqrt(1.0 + X * X);
              xt = sg * Cq * X / s1;
              xp = -sg * Cq / s1 * tq / s2;
              et = sg * Cx * tq / s1;
              ep = sg * Cx / s1 * X / s2;
            }
          }
          RC(z, e, l, q, 0, 0) = xt;
          RC(z, e, l, q, 0, 1) = xp;
          RC(z, e, l, q, 1, 0) = et;
          RC(z, e, l, q, 1, 1) = ep;
        }
      }
    }

  // Fold everything an edge value needs into one set of coefficients per ghost point.
  t.ew.assign((size_t)6 * 4 * 3 * 9 * n, 0.0);
  t.eg.assign((size_t)6 * 4 * 3 * 9 * 2 * n, 0.0);
  t.s0t.assign((size_t)6 * 4 * 3 * n, 0);
  t.egc.assign((size_t)6 * 4 * 3 * 9 * 4 * n, 0.0);
  for (int f = 0; f < 6; ++f)
    for (int e = 0; e < 4; ++e) {
      const EdgeRoute rt = kRoutes[f][e];
      const int kind = rt.src_face < 4 ? 0 : rt.src_face - 3;
      const size_t fe = (size_t)f * 4 + e;
      for (int l = 0; l < 3; ++l) {
        const int fixed = (rt.src_edge == kS || rt.src_edge == kW) ? l + 1 : n - 2 - l;
        for (int q = 0; q < n; ++q) {
          const int qs = rt.reversed ? n - 1 - q : q;
          const int s0 = t.s0[(size_t)l * n + qs];
          t.s0t[(fe * 3 + l) * n + q] = s0;
          const double c0 = ROT(rt.src_face, rt.src_edge, l, qs, 0);
          const double c1 = ROT(rt.src_face, rt.src_edge, l, qs, 1);
          for (int s = 0; s < 9; ++s) {
            const int ii = rt.src_edge <= kN ? s0 + s : fixed;
            const int jj = rt.src_edge <= kN ? fixed : s0 + s;
            const size_t p2 = (size_t)jj * n + ii;
            const double w = t.w9[((size_t)l * n + qs) * 9 + s];
            const double* a = &t.conv[(size_t)kind * 4 * P2];
            const size_t row = (fe * 3 + l) * 9 + s;
            t.ew[row * n + q] = w;
            t.eg[(row * 2 + 0) * n + q] = w * (c0 * a[0 * P2 + p2] + c1 * a[2 * P2 + p2]);
            t.eg[(row * 2 + 1) * n + q] = w * (c0 * a[1 * P2 + p2] + c1 * a[3 * P2 + p2]);
            for (int o = 0; o < 2; ++o) {
              const double ct = RC(rt.src_face, rt.src_edge, l, qs, o, 0), cp = RC(rt.src_face, rt.src_edge, l, qs, o, 1);
              t.egc[((row * 2 + o) * 2 + 0) * n + q] = w * (ct * a[0 * P2 + p2] + cp * a[2 * P2 + p2]);
              t.egc[((row * 2 + o) * 2 + 1) * n + q] = w * (ct * a[1 * P2 + p2] + cp * a[3 * P2 + p2]);
            }
          }
        }
      }
    }
  t.tspan.assign((size_t)6 * 4 * 3 * n * 2, 0);
  for (size_t fl = 0; fl < (size_t)6 * 4 * 3; ++fl)
    for (int u = 0; u < n; ++u) {
      int lo = n, hi = -1;
      for (int q = 0; q < n; ++q) {
        const int s0 = t.s0t[fl * n + q];
        if (u >= s0 && u <= s0 + 8) { lo = std::min(lo, q); hi = std::max(hi, q); }
      }
      if (hi < 0) lo = 0;
      t.tspan[(fl * n + u) * 2 + 0] = lo;
      t.tspan[(fl * n + u) * 2 + 1] = hi;
    }
  return SOLAR_OK;
}

}  // namespace solar
