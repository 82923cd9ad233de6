// kernels.cuh -- sm_100a kernels of the cubed-sphere time step.
//
// Device layout.  Every (run, face, field) volume is stored padded:
//     vol[k][row][col],  row = JOFF + j (j = -3 .. n+2),  col = IOFF + i (i = -3 .. n+2)
// with the interior i, j in [0, n) and a 3-deep ghost frame around it that holds the
// neighbouring faces' interpolated values (the reference's fp / fn halo arrays,
// derivative.f90:20, filter.f90:60).  The frame is rewritten before every consumer
// because its contents depend on the use (scalar halos for the pressure gradient and the
// filter, receiver-frame vector components for the divergence).  Corner cells outside
// both ranges are never read by a stencil.  Rows are padded so that the interior of
// every row starts on a 32-byte boundary.
//
// Buffers: A holds the state between steps, B is the stage ping-pong partner, W holds
// the 2N-RK register qw.  One step is
//     5 x [edge(rhs) ; stage]  (A->B, B->A, A->B, B->A, A->B)  then  edge(filter) ; filter (B->A)
// so the state returns to A and one captured graph serves every step.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace solar {

constexpr int IOFF = 8;   // interior column offset inside a padded row
constexpr int JOFF = 3;   // interior row offset inside a padded plane

// storage slots of the five reference fields (rho, v_xi, v_eta, v_r, p)
enum Field { kRho = 0, kVxi = 1, kVeta = 2, kVr = 3, kP = 4 };

struct Geom {
  int n, nr, nf;            // points per edge, radial points, stored fields
  int pitch, rows;          // padded row pitch and row count
  long long plane, vs;      // padded plane size; volume stride (per run/face/field)
  int nruns;
  int slot[5];              // slot of each reference field, -1 if not stored
  __host__ __device__ long long vol(int run, int face, int s) const {
    return ((long long)(run * 6 + face) * nf + s) * vs;
  }
  __host__ __device__ long long at(int k, int j, int i) const {
    return (long long)k * plane + (long long)(JOFF + j) * pitch + IOFF + i;
  }
};

struct EdgeRouteDev { int src_face, src_edge, reversed; };

// Scheme constants in constant memory (double and float copies).
__constant__ double cDrpD[4];
__constant__ double cBdyD[3][7];
__constant__ double cFiltD[4];
__constant__ double cFiltRD[6];
__constant__ float cDrpF[4];
__constant__ float cBdyF[3][7];
__constant__ float cFiltF[4];
__constant__ float cFiltRF[6];
__constant__ EdgeRouteDev cRoute[6][4];

template <typename T> struct Coef;
template <> struct Coef<double> {
  __device__ static double drp(int m) { return cDrpD[m]; }
  __device__ static double bdy(int r, int m) { return cBdyD[r][m]; }
  __device__ static double filt(int m) { return cFiltD[m]; }
  __device__ static double filtr(int m) { return cFiltRD[m]; }
};
template <> struct Coef<float> {
  __device__ static float drp(int m) { return cDrpF[m]; }
  __device__ static float bdy(int r, int m) { return cBdyF[r][m]; }
  __device__ static float filt(int m) { return cFiltF[m]; }
  __device__ static float filtr(int m) { return cFiltRF[m]; }
};

// ---------------------------------------------------------------------------------
// Edge (ghost) kernel: INTERPOLATE_ALONG_X/Y + TRANSFORM_VECTOR_BETWEEN_MESHES_DIV +
// the inter-zone exchange and its reversal, all in one pass.  One thread computes one
// ghost value (receiver face, edge, layer, k, position along the edge) by a 9-tap
// Lagrange sum over the source face's plane 1+layer / n-2-layer.
// mode 0: RHS halos -- p scalar on all edges; v_xi rotated on W/E; v_eta rotated on S/N.
// mode 1: filter halos -- every stored field, scalar, all edges (filter.f90:23-28).
template <typename T>
struct EdgeArgs {
  T* q;                     // buffer whose frames are filled (interior is the source)
  const T* w9;              // [3][n][9]
  const int* s0;            // [3][n]
  const T* conv;            // [3 kinds][4][n][n]
  const T* rot;             // [6][4][3][n][2]
  const int* active;        // per-run flag or nullptr
  Geom g;
  int mode;
};

template <typename T>
__global__ void __launch_bounds__(192) edge_kernel(const EdgeArgs<T> a) {
  const Geom& g = a.g;
  const int n = g.n;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;   // position along the edge
  const int l = threadIdx.y;                             // ghost layer 0..2
  const int k = blockIdx.y;
  const int z = blockIdx.z;                              // (run*6 + face)*4 + edge
  const int e = z & 3, face = (z >> 2) % 6, run = (z >> 2) / 6;
  if (t >= n) return;
  if (a.active && !a.active[run]) return;
  const EdgeRouteDev rt = cRoute[face][e];
  const int ts = rt.reversed ? n - 1 - t : t;
  const int s0 = a.s0[l * n + ts];
  const T* w = a.w9 + ((long long)l * n + ts) * 9;
  // source points: along i on row js (S/N strips) or along j on column is (W/E strips)
  const bool along_i = rt.src_edge <= 1;
  const int fixed = (rt.src_edge == 0 || rt.src_edge == 2) ? l + 1 : n - 2 - l;
  long long src_off[9];
  int src_p2[9];
#pragma unroll
  for (int s = 0; s < 9; ++s) {
    const int ii = along_i ? s0 + s : fixed;
    const int jj = along_i ? fixed : s0 + s;
    src_off[s] = g.at(k, jj, ii);
    src_p2[s] = jj * n + ii;
  }
  long long dst;
  if (e == 0) dst = g.at(k, -1 - l, t);
  else if (e == 1) dst = g.at(k, n + l, t);
  else if (e == 2) dst = g.at(k, t, -1 - l);
  else dst = g.at(k, t, n + l);

  auto scalar = [&](int slot) {
    const T* src = a.q + g.vol(run, rt.src_face, slot);
    T acc = T(0);
#pragma unroll
    for (int s = 0; s < 9; ++s) acc = fma(w[s], __ldg(src + src_off[s]), acc);
    a.q[g.vol(run, face, slot) + dst] = acc;
  };
  if (a.mode == 1) {
    for (int s = 0; s < g.nf; ++s) scalar(s);
    return;
  }
  scalar(g.slot[kP]);
  // vector component: v_xi for W/E receivers, v_eta for S/N receivers
  const T* vx = a.q + g.vol(run, rt.src_face, g.slot[kVxi]);
  const T* ve = a.q + g.vol(run, rt.src_face, g.slot[kVeta]);
  const int kind = rt.src_face < 4 ? 0 : rt.src_face - 3;
  const long long P2 = (long long)n * n;
  const T* cv = a.conv + (long long)kind * 4 * P2;
  T th = T(0), ph = T(0);
#pragma unroll
  for (int s = 0; s < 9; ++s) {
    const T x = __ldg(vx + src_off[s]), y = __ldg(ve + src_off[s]);
    const int p2 = src_p2[s];
    const T tht = fma(cv[p2], x, cv[P2 + p2] * y);
    const T pht = fma(cv[2 * P2 + p2], x, cv[3 * P2 + p2] * y);
    th = fma(w[s], tht, th);
    ph = fma(w[s], pht, ph);
  }
  const T* rc = a.rot + ((((long long)rt.src_face * 4 + rt.src_edge) * 3 + l) * n + ts) * 2;
  const int out_slot = (e >= 2) ? g.slot[kVxi] : g.slot[kVeta];
  a.q[g.vol(run, face, out_slot) + dst] = fma(rc[0], th, rc[1] * ph);
}

// ---------------------------------------------------------------------------------
// Stage kernel: COMPUTE_RHS (divergence, gradient, background terms) + BC_RHS + SPONGE
// + the 2N-RK update (timestep.f90:64-69) for one stage, fused.  A CTA owns a TX x TY
// column tile of one face and marches along k through its chunk.  xi/eta derivatives
// read shared-memory tiles of plane k with a 3-point halo (from the padded frame at the
// face edges); the radial derivative reads a 7-plane register window of the thread's own
// column, shifted as k advances and clamped at the two radial ends where the Tam-Dong
// one-sided rows apply (derivative.f90:704-754).
// MODE 0: RK update, stages 2-5 (reads qw).  MODE 1: RK update, stage 1 (qw = 0).
// MODE 2: write the raw COMPUTE_RHS into out.  MODE 3: write (grad_xi, grad_eta,
// grad_r, div) into the v_xi, v_eta, v_r, p slots of out.
template <typename T>
struct StageArgs {
  const T* qin;
  T* qout;
  T* qw;
  const T* rad;             // [kNumRadial][nr]
  const T* met;             // [kNumMetric][n][n]
  const T* c2;              // optional compact c^2 [face][k][j][i] (run-shared) or nullptr
  const int* active;
  Geom g;
  T dt, alpha, beta, inv_dxi;
  int kchunk;
};

// radial table rows (must match tables.h)
enum { rInvR = 0, rFacR, rRho0, rInvRho0, rC2Rho0, rDRho0, rG0Rho0, rRho0G0, rSigma, rCount };
enum { mD = 0, mXYD, mC, mXYC, mDivX, mDivY, mTX, mTY, mVol, mCount };

template <typename T, int TX, int TY, int MODE>
__global__ void __launch_bounds__(TX * TY) stage_kernel(const StageArgs<T> a) {
  const Geom& g = a.g;
  const int n = g.n, nr = g.nr;
  const int tiles_x = n / TX;
  const int i0 = (blockIdx.x % tiles_x) * TX, j0 = (blockIdx.x / tiles_x) * TY;
  const int rf = blockIdx.z, run = rf / 6, face = rf % 6;
  if (a.active && !a.active[run]) return;
  const int kb = blockIdx.y * a.kchunk;
  if (kb >= nr) return;
  const int ke = min(nr, kb + a.kchunk);
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i = i0 + tx, j = j0 + ty;

  __shared__ T sp[TY + 6][TX + 6];
  __shared__ T sx[TY][TX + 6];
  __shared__ T sy[TY + 6][TX];

  const int sP = g.slot[kP], sX = g.slot[kVxi], sY = g.slot[kVeta], sR = g.slot[kVr], sRho = g.slot[kRho];
  const T* qP = a.qin + g.vol(run, face, sP);
  const T* qX = a.qin + g.vol(run, face, sX);
  const T* qY = a.qin + g.vol(run, face, sY);
  const T* qR = a.qin + g.vol(run, face, sR);
  const T* qRho = sRho >= 0 ? a.qin + g.vol(run, face, sRho) : nullptr;

  const long long P2 = (long long)n * n;
  const int p2 = j * n + i;
  const T m_D = a.met[mD * P2 + p2], m_XYD = a.met[mXYD * P2 + p2];
  const T m_C = a.met[mC * P2 + p2], m_XYC = a.met[mXYC * P2 + p2];
  const T m_DivX = a.met[mDivX * P2 + p2], m_DivY = a.met[mDivY * P2 + p2];
  const T m_TX = a.met[mTX * P2 + p2], m_TY = a.met[mTY * P2 + p2];
  const T c1 = Coef<T>::drp(1), c2 = Coef<T>::drp(2), c3 = Coef<T>::drp(3);

  const long long own = g.at(0, j, i);
  auto clampk = [nr](int k) { return min(max(k - 3, 0), nr - 7); };
  T pw[7], vw[7];
  int ks = clampk(kb);
#pragma unroll
  for (int s = 0; s < 7; ++s) {
    pw[s] = qP[(long long)(ks + s) * g.plane + own];
    vw[s] = qR[(long long)(ks + s) * g.plane + own];
  }

  for (int k = kb; k < ke; ++k) {
    const int ksn = clampk(k);
    if (ksn != ks) {
#pragma unroll
      for (int s = 0; s < 6; ++s) { pw[s] = pw[s + 1]; vw[s] = vw[s + 1]; }
      ks = ksn;
      pw[6] = qP[(long long)(ks + 6) * g.plane + own];
      vw[6] = qR[(long long)(ks + 6) * g.plane + own];
    }
    const long long kp = (long long)k * g.plane;
    __syncthreads();
    for (int idx = tid; idx < (TY + 6) * (TX + 6); idx += TX * TY) {
      const int r = idx / (TX + 6), c = idx % (TX + 6);
      sp[r][c] = qP[kp + g.at(0, j0 - 3 + r, i0 - 3 + c)];
    }
    for (int idx = tid; idx < TY * (TX + 6); idx += TX * TY) {
      const int r = idx / (TX + 6), c = idx % (TX + 6);
      sx[r][c] = qX[kp + g.at(0, j0 + r, i0 - 3 + c)];
    }
    for (int idx = tid; idx < (TY + 6) * TX; idx += TX * TY) {
      const int r = idx / TX, c = idx % TX;
      sy[r][c] = qY[kp + g.at(0, j0 - 3 + r, i0 + c)];
    }
    __syncthreads();

    const T dpx = a.inv_dxi * (c1 * (sp[ty + 3][tx + 4] - sp[ty + 3][tx + 2]) +
                               c2 * (sp[ty + 3][tx + 5] - sp[ty + 3][tx + 1]) +
                               c3 * (sp[ty + 3][tx + 6] - sp[ty + 3][tx]));
    const T dpy = a.inv_dxi * (c1 * (sp[ty + 4][tx + 3] - sp[ty + 2][tx + 3]) +
                               c2 * (sp[ty + 5][tx + 3] - sp[ty + 1][tx + 3]) +
                               c3 * (sp[ty + 6][tx + 3] - sp[ty][tx + 3]));
    const T dvx = a.inv_dxi * (c1 * (sx[ty][tx + 4] - sx[ty][tx + 2]) +
                               c2 * (sx[ty][tx + 5] - sx[ty][tx + 1]) +
                               c3 * (sx[ty][tx + 6] - sx[ty][tx]));
    const T dvy = a.inv_dxi * (c1 * (sy[ty + 4][tx] - sy[ty + 2][tx]) +
                               c2 * (sy[ty + 5][tx] - sy[ty + 1][tx]) +
                               c3 * (sy[ty + 6][tx] - sy[ty][tx]));
    const T facr = a.rad[rFacR * nr + k];
    T dpr, dvr;
    if (k >= 3 && k <= nr - 4) {
      dpr = facr * (c1 * (pw[4] - pw[2]) + c2 * (pw[5] - pw[1]) + c3 * (pw[6] - pw[0]));
      dvr = facr * (c1 * (vw[4] - vw[2]) + c2 * (vw[5] - vw[1]) + c3 * (vw[6] - vw[0]));
    } else {
      const bool lo = k < 3;
      const int row = lo ? k : nr - 1 - k;
      T sp_ = T(0), sv_ = T(0);
#pragma unroll
      for (int s = 0; s < 7; ++s) {
        const T b = Coef<T>::bdy(row, lo ? s : 6 - s);
        sp_ = fma(b, pw[s], sp_);
        sv_ = fma(b, vw[s], sv_);
      }
      dpr = lo ? facr * sp_ : -facr * sp_;
      dvr = lo ? facr * sv_ : -facr * sv_;
    }
    const int off = k - ks;
    T vr = vw[0];
#pragma unroll
    for (int s = 1; s < 7; ++s) vr = (off == s) ? vw[s] : vr;
    const T p = sp[ty + 3][tx + 3];
    const T vxi = sx[ty][tx + 3];
    const T veta = sy[ty + 3][tx];

    const T invr = a.rad[rInvR * nr + k];
    const T gxi = invr * (m_D * dpx + m_XYD * dpy);
    const T geta = invr * (m_C * dpy + m_XYC * dpx);
    const T div = invr * (m_DivX * dvx + m_DivY * dvy - m_TX * vxi - m_TY * veta) + dvr + T(2) * vr * invr;
    const long long pt = kp + own;

    if (MODE == 3) {
      a.qout[g.vol(run, face, sX) + pt] = gxi;
      a.qout[g.vol(run, face, sY) + pt] = geta;
      a.qout[g.vol(run, face, sR) + pt] = dpr;
      a.qout[g.vol(run, face, sP) + pt] = div;
      continue;
    }
    const T rho0 = a.rad[rRho0 * nr + k], inv_rho0 = a.rad[rInvRho0 * nr + k];
    T c2rho0 = a.rad[rC2Rho0 * nr + k];
    if (a.c2) c2rho0 = a.c2[((long long)face * nr + k) * P2 + p2] * rho0;
    const T rho = qRho ? qRho[pt] : T(0);
    T r_rho = -rho0 * div - vr * a.rad[rDRho0 * nr + k];
    T r_vx = -gxi * inv_rho0;
    T r_ve = -geta * inv_rho0;
    T r_vr = -dpr * inv_rho0 - rho * a.rad[rG0Rho0 * nr + k];
    T r_p = -c2rho0 * div + a.rad[rRho0G0 * nr + k] * vr;
    if (MODE == 2) {
      if (qRho) a.qout[g.vol(run, face, sRho) + pt] = r_rho;
      a.qout[g.vol(run, face, sX) + pt] = r_vx;
      a.qout[g.vol(run, face, sY) + pt] = r_ve;
      a.qout[g.vol(run, face, sR) + pt] = r_vr;
      a.qout[g.vol(run, face, sP) + pt] = r_p;
      continue;
    }
    // BC_RHS (bc_acoustic_wave.f90:432-452) then SPONGE (sponge.f90:502-504)
    if (k == 0 || k == nr - 1) { r_rho = r_vx = r_ve = r_vr = r_p = T(0); }
    const T sig = a.rad[rSigma * nr + k];
    r_rho -= sig * rho;
    r_vr -= sig * vr;
    r_p -= sig * p;
    // qw = alpha qw + dt rhs ; q = q + beta qw   (timestep.f90:68-69)
    auto update = [&](int s, T q, T r) {
      T* W = a.qw + g.vol(run, face, s) + pt;
      const T w = (MODE == 1) ? a.dt * r : fma(a.alpha, *W, a.dt * r);
      *W = w;
      a.qout[g.vol(run, face, s) + pt] = fma(a.beta, w, q);
    };
    if (qRho) update(sRho, rho, r_rho);
    update(sX, vxi, r_vx);
    update(sY, veta, r_ve);
    update(sR, vr, r_vr);
    update(sP, p, r_p);
  }
}

// ---------------------------------------------------------------------------------
// Filter kernel: FILTER_EXP for one field (filter.f90:9-48): xi filter of q (with the
// q halos), eta filter of that (rows outside the face take the UNFILTERED q halo,
// filter.f90:43), 11-point radial filter of the result; the 5 end planes at each radial
// end become 0 (filter.f90:726-775).  A CTA owns a TX x TY column tile of one face and
// one field and marches through every k with an 11-deep register queue.
template <typename T>
struct FilterArgs {
  const T* qin;
  T* qout;
  const int* active;
  Geom g;
};

template <typename T, int TX, int TY>
__global__ void __launch_bounds__(TX * TY) filter_kernel(const FilterArgs<T> a) {
  const Geom& g = a.g;
  const int n = g.n, nr = g.nr;
  const int tiles_x = n / TX;
  const int i0 = (blockIdx.x % tiles_x) * TX, j0 = (blockIdx.x / tiles_x) * TY;
  const int s = blockIdx.y;                  // stored field
  const int rf = blockIdx.z, run = rf / 6, face = rf % 6;
  if (a.active && !a.active[run]) return;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i = i0 + tx, j = j0 + ty;
  __shared__ T sq[TY + 6][TX + 6];
  __shared__ T st[TY + 6][TX];
  const T* q = a.qin + g.vol(run, face, s);
  T* out = a.qout + g.vol(run, face, s);
  const long long own = g.at(0, j, i);
  const T f0 = Coef<T>::filt(0), f1 = Coef<T>::filt(1), f2 = Coef<T>::filt(2), f3 = Coef<T>::filt(3);
  T tq[11];
#pragma unroll
  for (int m = 0; m < 11; ++m) tq[m] = T(0);
  for (int k = 0; k < nr; ++k) {
    const long long kp = (long long)k * g.plane;
    __syncthreads();
    for (int idx = tid; idx < (TY + 6) * (TX + 6); idx += TX * TY) {
      const int r = idx / (TX + 6), c = idx % (TX + 6);
      sq[r][c] = q[kp + g.at(0, j0 - 3 + r, i0 - 3 + c)];
    }
    __syncthreads();
    for (int r = ty; r < TY + 6; r += TY) {
      const int jr = j0 - 3 + r;
      T v;
      if (jr < 0 || jr >= n) {
        v = sq[r][tx + 3];
      } else {
        v = f0 * sq[r][tx + 3] + f1 * (sq[r][tx + 2] + sq[r][tx + 4]) +
            f2 * (sq[r][tx + 1] + sq[r][tx + 5]) + f3 * (sq[r][tx] + sq[r][tx + 6]);
      }
      st[r][tx] = v;
    }
    __syncthreads();
    const T t2 = f0 * st[ty + 3][tx] + f1 * (st[ty + 2][tx] + st[ty + 4][tx]) +
                 f2 * (st[ty + 1][tx] + st[ty + 5][tx]) + f3 * (st[ty][tx] + st[ty + 6][tx]);
#pragma unroll
    for (int m = 0; m < 10; ++m) tq[m] = tq[m + 1];
    tq[10] = t2;
    if (k >= 10) {
      T v = Coef<T>::filtr(0) * tq[5];
#pragma unroll
      for (int m = 1; m <= 5; ++m) v += Coef<T>::filtr(m) * (tq[5 - m] + tq[5 + m]);
      out[(long long)(k - 5) * g.plane + own] = v;
    }
    if (k < 5 || k >= nr - 5) out[kp + own] = T(0);
  }
}

// ---------------------------------------------------------------------------------
// State transfer: six-zone Fortran-order FP64 arrays <-> padded device volumes.
// One launch moves one (face, reference field) volume.
template <typename T>
__global__ void unpack_kernel(const double* __restrict__ src, T* __restrict__ dst, Geom g) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long V = (long long)g.n * g.n * g.nr;
  if (idx >= V) return;
  const int i = idx % g.n, j = (idx / g.n) % g.n, k = idx / ((long long)g.n * g.n);
  dst[g.at(k, j, i)] = (T)src[idx];
}

template <typename T>
__global__ void pack_kernel(const T* __restrict__ src, double* __restrict__ dst, Geom g) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long V = (long long)g.n * g.n * g.nr;
  if (idx >= V) return;
  const int i = idx % g.n, j = (idx / g.n) % g.n, k = idx / ((long long)g.n * g.n);
  dst[idx] = src ? (double)src[g.at(k, j, i)] : 0.0;
}

// Pointwise BC_RHS / SPONGE on a device state (operator-level entry points).
template <typename T>
__global__ void bc_sponge_kernel(T* rhs, const T* q, const T* rad, Geom g, int run, int do_bc,
                                 int do_sponge) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long V = (long long)g.n * g.n * g.nr;
  if (idx >= 6 * V) return;
  const int face = idx / V;
  const long long l = idx % V;
  const int i = l % g.n, j = (l / g.n) % g.n, k = l / ((long long)g.n * g.n);
  const long long pt = g.at(k, j, i);
  for (int f = 0; f < 5; ++f) {
    const int s = g.slot[f];
    if (s < 0) continue;
    T* r = rhs + g.vol(run, face, s) + pt;
    if (do_bc && (k == 0 || k == g.nr - 1)) *r = T(0);
    if (do_sponge && (f == kRho || f == kVr || f == kP))
      *r -= rad[rSigma * g.nr + k] * q[g.vol(run, face, s) + pt];
  }
}

// Gaussian pressure pulse at the grid points x = r * unit(cube point of the face), added
// to one face's compact FP64 pressure volume p[k][j][i].
__global__ void gaussian_kernel(double* p, Geom g, int face, const double* tanx, const double* gr,
                                double x0, double y0, double z0, double width, double amp) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long V = (long long)g.n * g.n * g.nr;
  if (idx >= V) return;
  const int i = idx % g.n, j = (idx / g.n) % g.n, k = idx / ((long long)g.n * g.n);
  const double X = tanx[i], Y = tanx[j];
  double cx, cy, cz;
  switch (face) {
    case 0: cx = 1; cy = X; cz = Y; break;
    case 1: cx = -X; cy = 1; cz = Y; break;
    case 2: cx = -1; cy = -X; cz = Y; break;
    case 3: cx = X; cy = -1; cz = Y; break;
    case 4: cx = -Y; cy = X; cz = 1; break;
    default: cx = Y; cy = X; cz = -1; break;
  }
  const double s = gr[k] / sqrt(cx * cx + cy * cy + cz * cz);
  const double dx = s * cx - x0, dy = s * cy - y0, dz = s * cz - z0;
  p[idx] += amp * exp(-(dx * dx + dy * dy + dz * dz) / (2.0 * width * width));
}

// ---------------------------------------------------------------------------------
// FP64 reductions for norm / diagnostics.  Stage 1: one CTA per (face, k) plane writes
// 5 partials; stage 2: one CTA sums them in a fixed order (deterministic).
//   part[0] = sum f_sel^2, [1] = energy, [2] = mass, [3] = max |p|, [4] = non-finite count
template <typename T>
__global__ void reduce_plane_kernel(const T* q, Geom g, int run, int sel_slot, const double* rad64,
                                    const double* vol2, const double* drw, const double* c2_3d,
                                    double* part) {
  const int face = blockIdx.x / g.nr, k = blockIdx.x % g.nr;
  const int n = g.n;
  double acc[5] = {0, 0, 0, 0, 0};
  const double rho0 = rad64[rRho0 * g.nr + k];
  const double c2rho0 = rad64[rC2Rho0 * g.nr + k];
  const long long kp = (long long)k * g.plane;
  for (int p = threadIdx.x; p < n * n; p += blockDim.x) {
    const int i = p % n, j = p / n;
    const long long pt = kp + g.at(0, j, i);
    auto val = [&](int f) -> double {
      const int s = g.slot[f];
      return s < 0 ? 0.0 : (double)q[g.vol(run, face, s) + pt];
    };
    const double vx = val(kVxi), ve = val(kVeta), vr = val(kVr), pp = val(kP), rho = val(kRho);
    const double fs = sel_slot >= 0 ? (double)q[g.vol(run, face, sel_slot) + pt] : 0.0;
    const double dv = vol2[p] * drw[k];
    double cr = c2rho0;
    if (c2_3d) cr = c2_3d[((long long)face * g.nr + k) * n * n + p] * rho0;
    acc[0] += fs * fs;
    acc[1] += 0.5 * (rho0 * (vx * vx + ve * ve + vr * vr) + pp * pp / cr) * dv;
    acc[2] += rho * dv;
    acc[3] = fmax(acc[3], fabs(pp));
    if (!isfinite(vx) || !isfinite(ve) || !isfinite(vr) || !isfinite(pp) || !isfinite(rho)) acc[4] += 1.0;
  }
  __shared__ double red[5][256];
  for (int m = 0; m < 5; ++m) red[m][threadIdx.x] = acc[m];
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if ((int)threadIdx.x < st)
      for (int m = 0; m < 5; ++m)
        red[m][threadIdx.x] = (m == 3) ? fmax(red[m][threadIdx.x], red[m][threadIdx.x + st])
                                       : red[m][threadIdx.x] + red[m][threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int m = 0; m < 5; ++m) part[(long long)blockIdx.x * 5 + m] = red[m][0];
}

__global__ void reduce_final_kernel(const double* part, int nblocks, double* out) {
  __shared__ double red[5][256];
  double acc[5] = {0, 0, 0, 0, 0};
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
    for (int m = 0; m < 5; ++m)
      acc[m] = (m == 3) ? fmax(acc[m], part[(long long)b * 5 + m]) : acc[m] + part[(long long)b * 5 + m];
  for (int m = 0; m < 5; ++m) red[m][threadIdx.x] = acc[m];
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if ((int)threadIdx.x < st)
      for (int m = 0; m < 5; ++m)
        red[m][threadIdx.x] = (m == 3) ? fmax(red[m][threadIdx.x], red[m][threadIdx.x + st])
                                       : red[m][threadIdx.x] + red[m][threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int m = 0; m < 5; ++m) out[m] = red[m][0];
}

// Batched runs: per-step activity flags and step counters (kernel boundaries order them).
__global__ void batch_tick_kernel(const int* target, const int* done, int* active, int nruns) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < nruns) active[r] = done[r] < target[r] ? 1 : 0;
}
__global__ void batch_tock_kernel(const int* active, int* done, int nruns) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < nruns) done[r] += active[r];
}

}  // namespace solar
