// tables.h -- host-side FP64 setup of the cubed-sphere solver (product code).
//
// This is the part of the reference's driver that runs once before time stepping
// (cube.f90:35-51): SOLAR_DATA normalisation, SETUP_COORDINATES_METRICS_ALL and
// SETUP_LAGRANGE_INTERPOLANT, plus the receiver-frame rotation coefficients of
// TRANSFORM_VECTOR_BETWEEN_MESHES_DIV.  Everything is computed in double precision once
// and then uploaded (rounded once to float for the FP32 path).
#pragma once

#include <string>
#include <vector>

#include "../../include/solar_gpu.h"
#include "scheme.h"

namespace solar {

// Scheme constants.  The stencil weights are the published Tam & Webb DRP and Tam & Dong
// boundary stencils, the Vasilyev-Lund-Moin xi/eta filter, the Hanasoge-Duvall radial
// filter and the Cook-Cabot 2N-storage RK coefficients, as the reference lists them
// (header:40-55, 68-76, 99-105, 123-133).
extern const double kDrp[4];          // c0..c3 of the antisymmetric 7-point stencil
extern const double kBdy[3][7];       // one-sided rows for the first three points
// kFilt (f0..f3 of the symmetric 7-point filter) and kFiltR (f0..f5 of the symmetric
// 11-point radial filter) are in scheme.h.
extern const double kAlpha[5];
extern const double kBeta[5];

enum Edge { kS = 0, kN = 1, kW = 2, kE = 3 };

// Where the ghost strip of receiver face `face`, edge `edge` comes from: the source
// face's own edge strip, reversed along the edge or not.  One entry per (face, edge).
struct EdgeRoute { int src_face; int src_edge; int reversed; };
extern const EdgeRoute kRoutes[6][4];

// Radial table rows ([row][k]).
enum Radial {
  kInvR = 0,   // 1 / r_k
  kFacR,       // 1 / (dchi * dr/dchi_k)
  kRho0,
  kInvRho0,
  kC2Rho0,     // c^2 rho0
  kDRho0,      // d rho0 / dr by the radial stencil
  kG0Rho0,     // g0 / rho0
  kRho0G0,     // rho0 g0
  kSigma,      // sponge sigma_r
  kNumRadial
};

// Horizontal metric rows ([row][j][i]).
enum Metric {
  kMD = 0,     // D_j
  kMXYD,       // X Y / D_j
  kMC,         // C_i
  kMXYC,       // X Y / C_i
  kMDivX,      // delta / (C D) / C_i
  kMDivY,      // delta / (C D) / D_j
  kMTX,        // tan(xi_i) / D_j
  kMTY,        // tan(eta_j) / C_i
  kMVol,       // (1+X^2)(1+Y^2)/delta^(3/2) dxi deta   (area element on the unit sphere)
  kNumMetric
};

struct HostTables {
  int n = 0, nr = 0;
  double dxi = 0, dchi = 0;
  double dimc = 1;                                 // model row 1 sound speed (SOLAR_DATA's dimc)
  std::vector<double> gxi, gr, gdrdchi, tanx;     // 1-D grids (gxi == geta)
  std::vector<double> c2, rho0, g0;                // normalised radial background
  std::vector<double> radial;                      // [kNumRadial][nr]
  std::vector<double> metric;                      // [kNumMetric][n][n]
  std::vector<double> conv;                        // [3 kinds][4][n][n] (xi,eta)->(theta,phi)
  std::vector<double> w9;                          // [3 layers][n][9] window weights
  std::vector<int> s0;                             // [3 layers][n] window start
  std::vector<double> interpolant;                 // [3][n][9] reference layout (iter+4)
  std::vector<double> rot;                         // [6][4][3][n][2] receiver-frame (cth, cph)
  // Folded edge coefficients, indexed by the RECEIVING face / edge and stored with the
  // position along the edge fastest (t):
  //   scalar ghost  = sum_s ew[f][e][l][s][t] * f(source tap s)
  //   vector ghost  = sum_s eg[f][e][l][s][0][t] * v_xi(tap s) + eg[f][e][l][s][1][t] * v_eta(tap s)
  // (Lagrange weight x local->global conversion at the source point x receiver rotation);
  // tap s sits at position s0t[f][e][l][t] + s of the source line.
  std::vector<double> ew;                          // [6][4][3][9][n]
  std::vector<double> eg;                          // [6][4][3][9][2][n]
  std::vector<int> s0t;                            // [6][4][3][n]
  // Transposed exchange: the ghost points t whose 9 taps include source position u form a
  // contiguous range, tspan[f][e][l][u] = (first t, last t); (0, -1) when empty.
  std::vector<int> tspan;                          // [6][4][3][n][2]
  // COMPUTE_CURL's vector halos carry both receiver components:
  //   ghost_out = sum_s egc[f][e][l][s][out][in][t] * v_in(tap s),  out/in = (xi, eta)
  std::vector<double> egc;                         // [6][4][3][9][2][2][n]
  std::vector<double> dr_weight;                   // [nr] radial volume weight r^2 dr
};

// Builds every table from the descriptor.  Returns SOLAR_OK or SOLAR_ERR_ARG with `err`.
int build_tables(const solar_desc& d, HostTables& t, std::string& err);

}  // namespace solar
