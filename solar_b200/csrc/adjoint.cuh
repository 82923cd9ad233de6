// adjoint.cuh -- discrete adjoint of the time step (sm_100a).
//
// The forward step is linear in the state: per 2N-RK stage s (timestep.f90:64-69)
//     w_s = alpha_s w_{s-1} + dt L(q_{s-1}) ,   q_s = q_{s-1} + beta_s w_s
// with L = SPONGE o BC_RHS o COMPUTE_RHS, then q_{n+1} = F(q_5) (FILTER_EXP).  Its exact
// transpose, stage by stage in reverse, is
//     mu_s = lw_s + beta_s lq_s ;  lq_{s-1} = lq_s + dt L^T(mu_s) ;  lw_{s-1} = alpha_s mu_s
// and the gradient of a misfit with respect to a per-point sound-speed perturbation dc
// (c -> c + dc enters only r_p = -c^2 rho0 div v, compute_rhs_acoustic.f90:134) gathers
//     g += dt (-2 c rho0 div(v_{s-1})) mu_s^p            (0 on the BC planes).
// L^T is applied in three kernels:
//   adj_pre    pointwise: mu, the BC mask, the coefficient-weighted fields whose transposed
//              derivatives make up L^T, the pointwise terms, the sponge, lw and g;
//   adj_deriv  transposed derivatives: -D_xi and -D_eta with zero halos (the DRP stencil is
//              antisymmetric), the radial transpose written out row by row (one-sided rows
//              and the dr/dchi metric), evaluated on the interior and on the ghost frame --
//              the frame values are the adjoints of the neighbour faces' ghost values;
//   adj_edge   the transpose of the edge exchange: ghost adjoints scattered (atomic adds)
//              into the source faces' lines with the same folded coefficients.
// FILTER_EXP^T is the radial transpose, then eta, then xi, each with its ghost-frame
// adjoints, then the same scatter.
#pragma once

#include "kernels.cuh"

namespace solar {

template <typename T>
struct AdjArgs {
  const T* lq;        // lambda_q of the stage output (padded, interior)
  T* lw;              // lambda_w, updated in place
  T* lout;            // lambda_q of the stage input: interior + ghost-frame adjoints
  T* inter;           // 6 intermediate volumes per (run, face): X1 Y1 R1 X2 Y2 R2, zero frames
  const T* div;       // compact [run][face][k][j][i] divergence of the stage input (BC-masked)
  const T* c2;        // optional per-point c^2 [face][k][j][i] or nullptr (radial)
  double* grad;       // compact [run][face][k][j][i] gradient accumulator, or nullptr
  const T* rad;
  const T* met;
  Geom g;
  T alpha, beta, dt, inv_dxi;
  int keep;           // 1: lout = lq + dt L^T mu (RK adjoint); 0: lout = L^T mu (operator)
};

__device__ __forceinline__ long long inter_vol(const Geom& g, int run, int face, int m) {
  return ((long long)(run * 6 + face) * 6 + m) * g.vs;
}

template <typename T>
__global__ void adj_pre_kernel(const AdjArgs<T> a) {
  const Geom& g = a.g;
  const int n = g.n, nr = g.nr;
  const long long V = (long long)n * n * nr;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)g.nruns * 6 * V) return;
  const int rf = idx / V, run = rf / 6, face = rf % 6;
  const long long l = idx % V;
  const int i = l % n, j = (l / n) % n, k = l / ((long long)n * n);
  const long long pt = g.at(k, j, i);
  const long long P2 = (long long)n * n;
  const int p2 = j * n + i;
  T mu[5], muq[5];
#pragma unroll
  for (int f = 0; f < 5; ++f) {
    const int s = g.slot[f];
    if (s < 0) { mu[f] = muq[f] = T(0); continue; }
    const long long o = g.vol(run, face, s) + pt;
    const T lq = a.lq[o];
    muq[f] = lq;
    mu[f] = a.lw[o] + a.beta * lq;
    a.lw[o] = a.alpha * mu[f];
  }
  const bool bc = (k == 0 || k == nr - 1);
  T mp[5];
#pragma unroll
  for (int f = 0; f < 5; ++f) mp[f] = bc ? T(0) : mu[f];
  const T invr = a.rad[rInvR * nr + k], inv_rho0 = a.rad[rInvRho0 * nr + k], rho0 = a.rad[rRho0 * nr + k];
  const T c2rho0 = a.c2 ? a.c2[((long long)face * nr + k) * P2 + p2] * rho0 : a.rad[rC2Rho0 * nr + k];
  const T tD = a.met[mD * P2 + p2], tXYD = a.met[mXYD * P2 + p2], tC = a.met[mC * P2 + p2], tXYC = a.met[mXYC * P2 + p2];
  const T tDivX = a.met[mDivX * P2 + p2], tDivY = a.met[mDivY * P2 + p2], tTX = a.met[mTX * P2 + p2], tTY = a.met[mTY * P2 + p2];
  // r_vx = -inv_rho0 invr (D dpx + XY/D dpy),  r_ve = -inv_rho0 invr (C dpy + XY/C dpx),  r_vr = -inv_rho0 dpr - rho g0/rho0
  const T X1 = -invr * inv_rho0 * (tD * mp[kVxi] + tXYC * mp[kVeta]);
  const T Y1 = -invr * inv_rho0 * (tXYD * mp[kVxi] + tC * mp[kVeta]);
  const T R1 = -inv_rho0 * mp[kVr];
  // r_p = -c^2 rho0 div + rho0 g0 v_r ; r_rho = -rho0 div - v_r drho0
  const T e = -c2rho0 * mp[kP] - rho0 * mp[kRho];
  const T X2 = invr * tDivX * e, Y2 = invr * tDivY * e, R2 = e;
  T* I = a.inter;
  I[inter_vol(g, run, face, 0) + pt] = X1;
  I[inter_vol(g, run, face, 1) + pt] = Y1;
  I[inter_vol(g, run, face, 2) + pt] = R1;
  I[inter_vol(g, run, face, 3) + pt] = X2;
  I[inter_vol(g, run, face, 4) + pt] = Y2;
  I[inter_vol(g, run, face, 5) + pt] = R2;
  const T sig = a.rad[rSigma * nr + k];
  T pw[5];
  pw[kRho] = -a.rad[rG0Rho0 * nr + k] * mp[kVr] - sig * mu[kRho];
  pw[kVxi] = -invr * tTX * e;
  pw[kVeta] = -invr * tTY * e;
  pw[kVr] = T(2) * invr * e - a.rad[rDRho0 * nr + k] * mp[kRho] + a.rad[rRho0G0 * nr + k] * mp[kP] - sig * mu[kVr];
  pw[kP] = -sig * mu[kP];
#pragma unroll
  for (int f = 0; f < 5; ++f) {
    const int s = g.slot[f];
    if (s < 0) continue;
    a.lout[g.vol(run, face, s) + pt] = (a.keep ? muq[f] : T(0)) + a.dt * pw[f];
  }
  if (a.grad) {
    const long long gi = (long long)rf * V + l;
    const T c = sqrt(c2rho0 * inv_rho0);
    a.grad[gi] += (double)(a.dt * (T(-2) * c * rho0 * a.div[gi]) * mp[kP]);
  }
}

// Transposed derivatives, on interior points and ghost-frame points.  One thread per
// (run, face, k, row, column) of the extended face (corners skipped).
template <typename T>
__global__ void adj_deriv_kernel(const AdjArgs<T> a) {
  const Geom& g = a.g;
  const int n = g.n, nr = g.nr, ne = n + 6;
  const long long E = (long long)ne * ne * nr;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)g.nruns * 6 * E) return;
  const int rf = idx / E, run = rf / 6, face = rf % 6;
  const long long l = idx % E;
  const int i = (int)(l % ne) - 3, j = (int)((l / ne) % ne) - 3, k = (int)(l / ((long long)ne * ne));
  const bool iin = i >= 0 && i < n, jin = j >= 0 && j < n;
  if (!iin && !jin) return;                       // corner: never read by a stencil
  const T* X1 = a.inter + inter_vol(g, run, face, 0);
  const T* Y1 = a.inter + inter_vol(g, run, face, 1);
  const T* R1 = a.inter + inter_vol(g, run, face, 2);
  const T* X2 = a.inter + inter_vol(g, run, face, 3);
  const T* Y2 = a.inter + inter_vol(g, run, face, 4);
  const T* R2 = a.inter + inter_vol(g, run, face, 5);
  auto at = [&](const T* f, int kk, int jj, int ii) -> T {
    return (ii >= 0 && ii < n && jj >= 0 && jj < n) ? f[g.at(kk, jj, ii)] : T(0);
  };
  // -D_xi f and -D_eta f with zero halos (D^T of an antisymmetric stencil)
  auto mdx = [&](const T* f) {
    T s = T(0);
#pragma unroll
    for (int m = 1; m <= 3; ++m) s += Coef<T>::drp(m) * (at(f, k, j, i + m) - at(f, k, j, i - m));
    return -a.inv_dxi * s;
  };
  auto mdy = [&](const T* f) {
    T s = T(0);
#pragma unroll
    for (int m = 1; m <= 3; ++m) s += Coef<T>::drp(m) * (at(f, k, j + m, i) - at(f, k, j - m, i));
    return -a.inv_dxi * s;
  };
  const long long pt = g.at(k, j, i);
  const int sP = g.slot[kP], sX = g.slot[kVxi], sY = g.slot[kVeta], sR = g.slot[kVr];
  if (!iin) {        // W/E ghost columns: adjoints of p and v_xi ghost values
    a.lout[g.vol(run, face, sP) + pt] = a.dt * mdx(X1);
    a.lout[g.vol(run, face, sX) + pt] = a.dt * mdx(X2);
    return;
  }
  if (!jin) {        // S/N ghost rows: adjoints of p and v_eta ghost values
    a.lout[g.vol(run, face, sP) + pt] = a.dt * mdy(Y1);
    a.lout[g.vol(run, face, sY) + pt] = a.dt * mdy(Y2);
    return;
  }
  // radial transpose: (Dr^T f)_k = sum_kk Dr[kk][k] f_kk
  auto drt = [&](const T* f) {
    T s = T(0);
#pragma unroll
    for (int m = -3; m <= 3; ++m) {
      const int kk = k - m;                            // row kk reads plane kk + m = k
      if (m == 0 || kk < 3 || kk > nr - 4) continue;
      const T cm = m > 0 ? Coef<T>::drp(m) : -Coef<T>::drp(-m);
      s += a.rad[rFacR * nr + kk] * cm * f[g.at(kk, j, i)];
    }
    if (k <= 6)
      for (int kk = 0; kk < 3; ++kk) s += a.rad[rFacR * nr + kk] * Coef<T>::bdy(kk, k) * f[g.at(kk, j, i)];
    if (k >= nr - 7)
      for (int kk = nr - 3; kk < nr; ++kk)
        s -= a.rad[rFacR * nr + kk] * Coef<T>::bdy(nr - 1 - kk, 6 - (k - (nr - 7))) * f[g.at(kk, j, i)];
    return s;
  };
  a.lout[g.vol(run, face, sP) + pt] += a.dt * (mdx(X1) + mdy(Y1) + drt(R1));
  a.lout[g.vol(run, face, sX) + pt] += a.dt * mdx(X2);
  a.lout[g.vol(run, face, sY) + pt] += a.dt * mdy(Y2);
  a.lout[g.vol(run, face, sR) + pt] += a.dt * drt(R2);
}

// Transpose of the edge exchange: every ghost-frame adjoint of buffer `q` is scattered back
// onto the source lines of the neighbouring face.  mode 0: p scalar + the rotated vector
// component (v_xi on W/E, v_eta on S/N); mode 1: every stored field scalar.
template <typename T>
__global__ void adj_edge_kernel(T* q, const T* ew, const T* eg, const int* s0t, Geom g, int mode) {
  const int n = g.n;
  const long long total = (long long)g.nruns * 24 * 3 * n * g.nr;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const int t = idx % n;
  long long r = idx / n;
  const int l = r % 3; r /= 3;
  const int k = r % g.nr; r /= g.nr;
  const int fe = r % 24, run = (int)(r / 24);
  const int face = fe >> 2, e = fe & 3;
  const EdgeRouteDev rt = cRoute[face][e];
  const bool along_i = rt.src_edge <= 1;
  const int fixed = (rt.src_edge == 0 || rt.src_edge == 2) ? l + 1 : n - 2 - l;
  const long long crow = ((long long)fe * 3 + l) * 9;
  const int s0 = s0t[((long long)fe * 3 + l) * n + t];
  long long dst;
  if (e == 0) dst = g.at(k, -1 - l, t);
  else if (e == 1) dst = g.at(k, n + l, t);
  else if (e == 2) dst = g.at(k, t, -1 - l);
  else dst = g.at(k, t, n + l);
  auto src_at = [&](int s) {
    const int ii = along_i ? s0 + s : fixed, jj = along_i ? fixed : s0 + s;
    return g.at(k, jj, ii);
  };
  if (mode == 1) {
    for (int sl = 0; sl < g.nf; ++sl) {
      const T gv = q[g.vol(run, face, sl) + dst];
      T* dstv = q + g.vol(run, rt.src_face, sl);
      for (int s = 0; s < 9; ++s) atomicAdd(dstv + src_at(s), ew[(crow + s) * n + t] * gv);
    }
    return;
  }
  const T gp = q[g.vol(run, face, g.slot[kP]) + dst];
  const T gv = q[g.vol(run, face, e >= 2 ? g.slot[kVxi] : g.slot[kVeta]) + dst];
  T* pp = q + g.vol(run, rt.src_face, g.slot[kP]);
  T* px = q + g.vol(run, rt.src_face, g.slot[kVxi]);
  T* py = q + g.vol(run, rt.src_face, g.slot[kVeta]);
  for (int s = 0; s < 9; ++s) {
    const long long o = src_at(s);
    atomicAdd(pp + o, ew[(crow + s) * n + t] * gp);
    atomicAdd(px + o, eg[((crow + s) * 2 + 0) * n + t] * gv);
    atomicAdd(py + o, eg[((crow + s) * 2 + 1) * n + t] * gv);
  }
}

// FILTER_R^T for every stored field: u_m = sum over output planes k in [5, nr-6] of
// fr_{|k-m|} lam_k (the end planes of the forward output are constant zeros).
template <typename T>
__global__ void adj_filter_r_kernel(const T* lam, T* u, Geom g) {
  const int n = g.n, nr = g.nr;
  const long long V = (long long)n * n * nr;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)g.nruns * 6 * g.nf * V) return;
  const long long vsel = idx / V;                      // (run*6 + face)*nf + slot
  const long long l = idx % V;
  const int i = l % n, j = (l / n) % n, m = l / ((long long)n * n);
  const T* L = lam + vsel * g.vs;
  T s = T(0);
  for (int d = -5; d <= 5; ++d) {
    const int k = m + d;
    if (k < 5 || k > nr - 6) continue;
    s += Coef<T>::filtr(d < 0 ? -d : d) * L[g.at(k, j, i)];
  }
  u[vsel * g.vs + g.at(m, j, i)] = s;
}

// FILTER_ETA^T (dir 1) or FILTER_XI^T (dir 0) with zero halos, evaluated on the interior and
// on the ghost rows (eta) / columns (xi) of the face.  Interior results go to `out`'s
// interior; ghost results are the adjoints of the (unfiltered) halo values and go to
// `frame`'s frame.
template <typename T>
__global__ void adj_filter_dir_kernel(const T* in, T* out, T* frame, Geom g, int dir) {
  const int n = g.n, nr = g.nr, ne = n + 6;
  const long long E = (long long)ne * n * nr;          // along-direction extended x other
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)g.nruns * 6 * g.nf * E) return;
  const long long vsel = idx / E;
  const long long l = idx % E;
  const int a_ = (int)(l % ne) - 3;                     // position along the filter direction
  const int b_ = (int)((l / ne) % n);                   // the other in-face coordinate
  const int k = (int)(l / ((long long)ne * n));
  const T* f = in + vsel * g.vs;
  auto val = [&](int aa) -> T {
    if (aa < 0 || aa >= n) return T(0);
    return dir ? f[g.at(k, aa, b_)] : f[g.at(k, b_, aa)];
  };
  T s = Coef<T>::filt(0) * val(a_);
#pragma unroll
  for (int m = 1; m <= 3; ++m) s += Coef<T>::filt(m) * (val(a_ - m) + val(a_ + m));
  const long long pt = dir ? g.at(k, a_, b_) : g.at(k, b_, a_);
  if (a_ >= 0 && a_ < n) out[vsel * g.vs + pt] = s;
  else frame[vsel * g.vs + pt] = s;
}

// Receivers: p sampled with trilinear weights over the 8 grid points around each receiver
// on its face.  rec_off[r*8+c] is the padded-buffer offset of corner c (p slot, run 0) and
// rec_w[r*8+c] its weight.  inject_kernel is the transpose of sample_kernel.
template <typename T>
__global__ void sample_kernel(const T* q, const long long* rec_off, const double* rec_w, int nrec, double* out) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrec) return;
  double s = 0.0;
  for (int c = 0; c < 8; ++c) s += rec_w[r * 8 + c] * (double)q[rec_off[r * 8 + c]];
  out[r] = s;
}

template <typename T>
__global__ void inject_kernel(T* lam, const long long* rec_off, const double* rec_w, int nrec, const double* res) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrec) return;
  for (int c = 0; c < 8; ++c) atomicAdd(lam + rec_off[r * 8 + c], (T)(rec_w[r * 8 + c] * res[r]));
}

// One slot of a padded buffer (run 0, all faces) -> compact [face][k][j][i].
template <typename T>
__global__ void gather_slot_kernel(const T* buf, int slot, T* dst, Geom g) {
  const long long V = (long long)g.n * g.n * g.nr;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= 6 * V) return;
  const int face = idx / V;
  const long long l = idx % V;
  const int i = l % g.n, j = (l / g.n) % g.n, k = l / ((long long)g.n * g.n);
  dst[idx] = buf[g.vol(0, face, slot) + g.at(k, j, i)];
}

}  // namespace solar
