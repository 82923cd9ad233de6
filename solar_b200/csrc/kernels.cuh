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

#include "tma.cuh"

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
// Edge (ghost) kernel: INTERPOLATE_ALONG_X/Y + TRANSFORM_VECTOR_BETWEEN_MESHES_DIV + the
// inter-zone exchange and its reversal, in one pass.  Each thread owns one ghost point
// (receiver face, edge, layer, position along the edge) and walks a chunk of radial planes.
// Its 9 source points and coefficients are loaded once: the scalar weights are the
// Lagrange weights; the vector coefficients fold the Lagrange weight, the source face's
// (xi,eta)->(theta,phi) conversion and the receiver-frame rotation into one pair per tap.
// mode 0: RHS halos -- p scalar on all edges; v_xi on W/E and v_eta on S/N, rotated.
// mode 1: filter halos -- every stored field, scalar, all edges (filter.f90:23-28).
template <typename T>
struct EdgeArgs {
  T* q;                     // buffer whose frames are filled (its interior is the source)
  const T* ew;              // [6][4][3][n][9]
  const T* eg;              // [6][4][3][n][9][2]
  const int* esrc;          // [6][4][3][n][9]  source point j*n + i
  const int* active;        // per-run flag or nullptr
  Geom g;
  int mode;
  int kchunk;
};

template <typename T>
__global__ void __launch_bounds__(192) edge_kernel(const EdgeArgs<T> a) {
  const Geom& g = a.g;
  const int n = g.n;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;   // position along the edge
  const int l = threadIdx.y;                             // ghost layer 0..2
  const int z = blockIdx.z;                              // (run*6 + face)*4 + edge
  const int e = z & 3, face = (z >> 2) % 6, run = (z >> 2) / 6;
  if (t >= n) return;
  if (a.active && !a.active[run]) return;
  const int kb = blockIdx.y * a.kchunk;
  const int ke = min(g.nr, kb + a.kchunk);
  const EdgeRouteDev rt = cRoute[face][e];
  const long long row = ((((long long)face * 4 + e) * 3 + l) * n + t) * 9;
  int off[9];
  T w[9];
#pragma unroll
  for (int s = 0; s < 9; ++s) {
    const int p2 = a.esrc[row + s];
    off[s] = (JOFF + p2 / n) * g.pitch + IOFF + p2 % n;
    w[s] = a.ew[row + s];
  }
  int dst;
  if (e == 0) dst = (JOFF - 1 - l) * g.pitch + IOFF + t;
  else if (e == 1) dst = (JOFF + n + l) * g.pitch + IOFF + t;
  else if (e == 2) dst = (JOFF + t) * g.pitch + IOFF - 1 - l;
  else dst = (JOFF + t) * g.pitch + IOFF + n + l;
  if (a.mode == 1) {
    for (int s = 0; s < g.nf; ++s) {
      const T* src = a.q + g.vol(run, rt.src_face, s);
      T* out = a.q + g.vol(run, face, s);
      for (int k = kb; k < ke; ++k) {
        const long long kp = (long long)k * g.plane;
        T acc = T(0);
#pragma unroll
        for (int m = 0; m < 9; ++m) acc = fma(w[m], __ldg(src + kp + off[m]), acc);
        out[kp + dst] = acc;
      }
    }
    return;
  }
  T gx[9], gy[9];
#pragma unroll
  for (int s = 0; s < 9; ++s) {
    gx[s] = a.eg[(row + s) * 2 + 0];
    gy[s] = a.eg[(row + s) * 2 + 1];
  }
  const T* sp = a.q + g.vol(run, rt.src_face, g.slot[kP]);
  const T* sx = a.q + g.vol(run, rt.src_face, g.slot[kVxi]);
  const T* sy = a.q + g.vol(run, rt.src_face, g.slot[kVeta]);
  T* op = a.q + g.vol(run, face, g.slot[kP]);
  T* ov = a.q + g.vol(run, face, (e >= 2) ? g.slot[kVxi] : g.slot[kVeta]);
#pragma unroll 2
  for (int k = kb; k < ke; ++k) {
    const long long kp = (long long)k * g.plane;
    T ap = T(0), av = T(0);
#pragma unroll
    for (int m = 0; m < 9; ++m) {
      ap = fma(w[m], __ldg(sp + kp + off[m]), ap);
      av = fma(gx[m], __ldg(sx + kp + off[m]), av);
      av = fma(gy[m], __ldg(sy + kp + off[m]), av);
    }
    op[kp + dst] = ap;
    ov[kp + dst] = av;
  }
}

// radial table rows (must match tables.h)
enum { rInvR = 0, rFacR, rRho0, rInvRho0, rC2Rho0, rDRho0, rG0Rho0, rRho0G0, rSigma, rCount };
enum { mD = 0, mXYD, mC, mXYC, mDivX, mDivY, mTX, mTY, mVol, mCount };

// ---------------------------------------------------------------------------------
// Stage kernel: COMPUTE_RHS (divergence, gradient, background terms) + BC_RHS + SPONGE
// + the 2N-RK update (timestep.f90:64-69) for one stage, fused.  A CTA owns a TX x TY
// column tile of one face and marches along k through its chunk of planes.
//
// Planes stream in through TMA tile loads into two shared-memory rings, each slot
// guarded by an mbarrier:
//   lead ring (kLead slots): the p tile with a 3-point halo and the v_r tile of plane m.
//     Plane m is needed from iteration m-3 (own values enter the 7-deep radial register
//     windows of p and v_r) until iteration m (xi/eta derivatives of p).
//   tile ring (kTile slots): v_xi with its xi halo, v_eta with its eta halo, rho and the
//     RK registers qw of plane k, needed at iteration k only.
// Thread 0 refills a slot right after the CTA barrier that closes the iteration using it,
// so up to kLead-4 lead planes and kTile-1 tile planes are in flight while a plane is
// computed.  The radial window is clamped at the two ends of the shell, where the
// Tam-Dong one-sided rows apply (derivative.f90:704-754).
// MODE 0: RK update, stages 2-5 (reads qw).  MODE 1: RK update, stage 1 (qw = 0).
// MODE 2: write the raw COMPUTE_RHS into qout.  MODE 3: write (grad_xi, grad_eta,
// grad_r, div) into the v_xi, v_eta, v_r, p slots of qout.
constexpr int kLead = 8;
constexpr int kTile = 3;

template <typename T>
struct StageArgs {
  CUtensorMap mP;           // input buffer, box (TX+8) x (TY+6)
  CUtensorMap mX;           // input buffer, box (TX+8) x TY
  CUtensorMap mY;           // input buffer, box TX x (TY+6)
  CUtensorMap mO;           // input buffer, box TX x TY
  CUtensorMap mW;           // qw buffer,    box TX x TY
  T* qout;
  T* qw;
  const T* rad;             // [kNumRadial][nr]
  const T* met;             // [kNumMetric][n][n]
  const T* c2;              // optional compact c^2 [face][k][j][i] (run-shared) or nullptr
  const int* active;
  int* err;
  Geom g;
  T dt, alpha, beta, inv_dxi;
  int kchunk;
};

__host__ __device__ constexpr size_t align128(size_t b) { return (b + 127) / 128 * 128; }

template <typename T, int TX, int TY>
struct StageLayout {
  static constexpr int PB = (TX + 8) * (TY + 6), XB = (TX + 8) * TY, YB = TX * (TY + 6), OB = TX * TY;
  static constexpr size_t P_BYTES = align128(PB * sizeof(T));
  static constexpr size_t X_BYTES = align128(XB * sizeof(T));
  static constexpr size_t Y_BYTES = align128(YB * sizeof(T));
  static constexpr size_t O_BYTES = align128(OB * sizeof(T));
  static constexpr size_t LEAD = P_BYTES + O_BYTES;                    // p box + v_r
  static constexpr size_t TILE = X_BYTES + Y_BYTES + 6 * O_BYTES;     // v_xi, v_eta, rho, 5 qw
  static constexpr size_t BAR = kLead * LEAD + kTile * TILE;
  static constexpr size_t TOTAL = BAR + (kLead + kTile) * sizeof(uint64_t);
};

template <typename T, int TX, int TY, int MODE>
__global__ void __launch_bounds__(TX * TY, sizeof(T) == 8 ? 2 : 3) stage_kernel(const __grid_constant__ StageArgs<T> a) {
  using L = StageLayout<T, TX, TY>;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L::BAR);
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
  const int sP = g.slot[kP], sX = g.slot[kVxi], sY = g.slot[kVeta], sR = g.slot[kVr], sRho = g.slot[kRho];
  const bool has_rho = sRho >= 0 && MODE != 3;
  const int zbase = (run * 6 + face) * g.nf;   // plane index of (slot s, k) = (zbase + s) * nr + k
  auto clampk = [nr](int k) { return min(max(k - 3, 0), nr - 7); };
  const int m_lo = clampk(kb), m_hi = clampk(ke - 1) + 6;

  auto leadP = [&](int m) { return reinterpret_cast<T*>(smem + ((m - m_lo) % kLead) * L::LEAD); };
  auto leadR = [&](int m) { return reinterpret_cast<T*>(smem + ((m - m_lo) % kLead) * L::LEAD + L::P_BYTES); };
  auto tileBase = [&](int k) { return smem + kLead * L::LEAD + ((k - kb) % kTile) * L::TILE; };
  auto tileX = [&](int k) { return reinterpret_cast<T*>(tileBase(k)); };
  auto tileY = [&](int k) { return reinterpret_cast<T*>(tileBase(k) + L::X_BYTES); };
  auto tileO = [&](int k, int q) { return reinterpret_cast<T*>(tileBase(k) + L::X_BYTES + L::Y_BYTES + q * L::O_BYTES); };
  uint64_t* barL = bars;
  uint64_t* barT = bars + kLead;

  const int xP = IOFF + i0 - 4, yP = JOFF + j0 - 3;   // p / v_xi boxes start 4 columns left
  const int xO = IOFF + i0, yO = JOFF + j0;
  auto issue_lead = [&](int m) {
    uint64_t* b = &barL[(m - m_lo) % kLead];
    mbar_expect_tx(b, (L::PB + L::OB) * sizeof(T));
    tma_load_3d(leadP(m), &a.mP, xP, yP, (zbase + sP) * nr + m, b);
    tma_load_3d(leadR(m), &a.mO, xO, yO, (zbase + sR) * nr + m, b);
  };
  auto issue_tile = [&](int k) {
    uint64_t* b = &barT[(k - kb) % kTile];
    uint32_t bytes = (L::XB + L::YB) * sizeof(T);
    if (has_rho) bytes += L::OB * sizeof(T);
    if (MODE == 0) bytes += g.nf * L::OB * sizeof(T);
    mbar_expect_tx(b, bytes);
    tma_load_3d(tileX(k), &a.mX, xP, yO, (zbase + sX) * nr + k, b);
    tma_load_3d(tileY(k), &a.mY, xO, yP, (zbase + sY) * nr + k, b);
    if (has_rho) tma_load_3d(tileO(k, 0), &a.mO, xO, yO, (zbase + sRho) * nr + k, b);
    if (MODE == 0)
      for (int s = 0; s < g.nf; ++s) tma_load_3d(tileO(k, 1 + s), &a.mW, xO, yO, (zbase + s) * nr + k, b);
  };

  if (tid == 0) {
    for (int q = 0; q < kLead + kTile; ++q) mbar_init(&bars[q], 1);
    mbar_fence_init();
  }
  __syncthreads();
  int m_issued = m_lo;
  if (tid == 0) {
    tma_prefetch_desc(&a.mP);
    for (; m_issued <= min(m_lo + kLead - 1, m_hi); ++m_issued) issue_lead(m_issued);
    for (int k = kb; k < min(kb + kTile, ke); ++k) issue_tile(k);
  }

  const long long P2 = (long long)n * n;
  const int p2 = j * n + i;
  const T m_D = a.met[mD * P2 + p2], m_XYD = a.met[mXYD * P2 + p2];
  const T m_C = a.met[mC * P2 + p2], m_XYC = a.met[mXYC * P2 + p2];
  const T m_DivX = a.met[mDivX * P2 + p2], m_DivY = a.met[mDivY * P2 + p2];
  const T m_TX = a.met[mTX * P2 + p2], m_TY = a.met[mTY * P2 + p2];
  const T c1 = Coef<T>::drp(1), c2 = Coef<T>::drp(2), c3 = Coef<T>::drp(3);
  const long long own = g.at(0, j, i);
  constexpr int PW = TX + 8;
  const int pc = (ty + 3) * PW + tx + 4;              // own point inside the p box

  T pw[7], vw[7];
#pragma unroll
  for (int s = 0; s < 7; ++s) { pw[s] = T(0); vw[s] = T(0); }
  int mq = m_lo;
  bool ok = true;
  for (int k = kb; k < ke; ++k) {
    const int ks = clampk(k);
    for (; mq <= ks + 6; ++mq) {
      ok &= mbar_wait(&barL[(mq - m_lo) % kLead], ((mq - m_lo) / kLead) & 1, a.err, 1);
#pragma unroll
      for (int s = 0; s < 6; ++s) { pw[s] = pw[s + 1]; vw[s] = vw[s + 1]; }
      pw[6] = leadP(mq)[pc];
      vw[6] = leadR(mq)[ty * TX + tx];
    }
    ok &= mbar_wait(&barT[(k - kb) % kTile], ((k - kb) / kTile) & 1, a.err, 2);
    const T* sp = leadP(k);
    const T* sx = tileX(k);
    const T* sy = tileY(k);
    const T dpx = a.inv_dxi * (c1 * (sp[pc + 1] - sp[pc - 1]) + c2 * (sp[pc + 2] - sp[pc - 2]) +
                               c3 * (sp[pc + 3] - sp[pc - 3]));
    const T dpy = a.inv_dxi * (c1 * (sp[pc + PW] - sp[pc - PW]) + c2 * (sp[pc + 2 * PW] - sp[pc - 2 * PW]) +
                               c3 * (sp[pc + 3 * PW] - sp[pc - 3 * PW]));
    const int xc = ty * PW + tx + 4;
    const T dvx = a.inv_dxi * (c1 * (sx[xc + 1] - sx[xc - 1]) + c2 * (sx[xc + 2] - sx[xc - 2]) +
                               c3 * (sx[xc + 3] - sx[xc - 3]));
    const int yc = (ty + 3) * TX + tx;
    const T dvy = a.inv_dxi * (c1 * (sy[yc + TX] - sy[yc - TX]) + c2 * (sy[yc + 2 * TX] - sy[yc - 2 * TX]) +
                               c3 * (sy[yc + 3 * TX] - sy[yc - 3 * TX]));
    const T facr = a.rad[rFacR * nr + k];
    T dpr, dvr;
    if (k >= 3 && k <= nr - 4) {
      dpr = facr * (c1 * (pw[4] - pw[2]) + c2 * (pw[5] - pw[1]) + c3 * (pw[6] - pw[0]));
      dvr = facr * (c1 * (vw[4] - vw[2]) + c2 * (vw[5] - vw[1]) + c3 * (vw[6] - vw[0]));
    } else {
      const bool lo = k < 3;
      const int brow = lo ? k : nr - 1 - k;
      T a_ = T(0), b_ = T(0);
#pragma unroll
      for (int s = 0; s < 7; ++s) {
        const T b = Coef<T>::bdy(brow, lo ? s : 6 - s);
        a_ = fma(b, pw[s], a_);
        b_ = fma(b, vw[s], b_);
      }
      dpr = lo ? facr * a_ : -facr * a_;
      dvr = lo ? facr * b_ : -facr * b_;
    }
    const int offk = k - ks;
    T vr = vw[0];
#pragma unroll
    for (int s = 1; s < 7; ++s) vr = (offk == s) ? vw[s] : vr;
    const T p = sp[pc];
    const T vxi = sx[xc];
    const T veta = sy[yc];
    const T invr = a.rad[rInvR * nr + k];
    const T gxi = invr * (m_D * dpx + m_XYD * dpy);
    const T geta = invr * (m_C * dpy + m_XYC * dpx);
    const T div = invr * (m_DivX * dvx + m_DivY * dvy - m_TX * vxi - m_TY * veta) + dvr + T(2) * vr * invr;
    const long long pt = (long long)k * g.plane + own;
    if (MODE == 3) {
      a.qout[g.vol(run, face, sX) + pt] = gxi;
      a.qout[g.vol(run, face, sY) + pt] = geta;
      a.qout[g.vol(run, face, sR) + pt] = dpr;
      a.qout[g.vol(run, face, sP) + pt] = div;
    } else {
      const T rho0 = a.rad[rRho0 * nr + k], inv_rho0 = a.rad[rInvRho0 * nr + k];
      T c2rho0 = a.rad[rC2Rho0 * nr + k];
      if (a.c2) c2rho0 = a.c2[((long long)face * nr + k) * P2 + p2] * rho0;
      const int oc = ty * TX + tx;
      const T rho = has_rho ? tileO(k, 0)[oc] : T(0);
      T r_rho = -rho0 * div - vr * a.rad[rDRho0 * nr + k];
      T r_vx = -gxi * inv_rho0;
      T r_ve = -geta * inv_rho0;
      T r_vr = -dpr * inv_rho0 - rho * a.rad[rG0Rho0 * nr + k];
      T r_p = -c2rho0 * div + a.rad[rRho0G0 * nr + k] * vr;
      if (MODE == 2) {
        if (has_rho) a.qout[g.vol(run, face, sRho) + pt] = r_rho;
        a.qout[g.vol(run, face, sX) + pt] = r_vx;
        a.qout[g.vol(run, face, sY) + pt] = r_ve;
        a.qout[g.vol(run, face, sR) + pt] = r_vr;
        a.qout[g.vol(run, face, sP) + pt] = r_p;
      } else {
        // BC_RHS (bc_acoustic_wave.f90:432-452) then SPONGE (sponge.f90:502-504)
        if (k == 0 || k == nr - 1) { r_rho = r_vx = r_ve = r_vr = r_p = T(0); }
        const T sig = a.rad[rSigma * nr + k];
        r_rho -= sig * rho;
        r_vr -= sig * vr;
        r_p -= sig * p;
        // qw = alpha qw + dt rhs ; q = q + beta qw   (timestep.f90:68-69)
        auto update = [&](int s, T q, T r) {
          const T w = (MODE == 1) ? a.dt * r : fma(a.alpha, tileO(k, 1 + s)[oc], a.dt * r);
          a.qw[g.vol(run, face, s) + pt] = w;
          a.qout[g.vol(run, face, s) + pt] = fma(a.beta, w, q);
        };
        if (has_rho) update(sRho, rho, r_rho);
        update(sX, vxi, r_vx);
        update(sY, veta, r_ve);
        update(sR, vr, r_vr);
        update(sP, p, r_p);
      }
    }
    // every thread is done with lead plane k and tile plane k: refill their slots
    if (__syncthreads_or(!ok)) break;
    if (tid == 0) {
      if (k + kTile < ke) issue_tile(k + kTile);
      for (; m_issued <= min(k + kLead, m_hi); ++m_issued) issue_lead(m_issued);
    }
  }
  if (!ok && tid == 0) {
    // a wait gave up: give copies still in flight a bounded time to land before exit
    for (int q = 0; q < 1000; ++q) __nanosleep(1000);
  }
}

// ---------------------------------------------------------------------------------
// Filter kernel: FILTER_EXP for one field (filter.f90:9-48): xi filter of q (with the
// q halos), eta filter of that (rows outside the face take the UNFILTERED q halo,
// filter.f90:43), 11-point radial filter of the result; the 5 end planes at each radial
// end become 0 (filter.f90:726-775).  A CTA owns a TX x TY column tile of one face and
// one field and streams every plane through a kFilt-deep TMA ring, keeping the last 11
// eta-filtered values of its column in registers.
constexpr int kFiltRing = 4;

template <typename T>
struct FilterArgs {
  CUtensorMap mP;           // input buffer, box (TX+8) x (TY+6)
  T* qout;
  const int* active;
  int* err;
  Geom g;
};

template <typename T, int TX, int TY>
struct FilterLayout {
  static constexpr int PB = (TX + 8) * (TY + 6), SB = (TY + 6) * TX;
  static constexpr size_t P_BYTES = align128(PB * sizeof(T));
  static constexpr size_t S_BYTES = align128(SB * sizeof(T));
  static constexpr size_t BAR = kFiltRing * P_BYTES + 2 * S_BYTES;
  static constexpr size_t TOTAL = BAR + kFiltRing * sizeof(uint64_t);
};

template <typename T, int TX, int TY>
__global__ void __launch_bounds__(TX * TY) filter_kernel(const __grid_constant__ FilterArgs<T> a) {
  using L = FilterLayout<T, TX, TY>;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L::BAR);
  const Geom& g = a.g;
  const int n = g.n, nr = g.nr;
  const int tiles_x = n / TX;
  const int i0 = (blockIdx.x % tiles_x) * TX, j0 = (blockIdx.x / tiles_x) * TY;
  const int s = blockIdx.y;                  // stored field
  const int rf = blockIdx.z, run = rf / 6, face = rf % 6;
  if (a.active && !a.active[run]) return;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i = i0 + tx, j = j0 + ty;
  constexpr int PW = TX + 8;
  auto box = [&](int k) { return reinterpret_cast<const T*>(smem + (k % kFiltRing) * L::P_BYTES); };
  auto st = [&](int k) { return reinterpret_cast<T*>(smem + kFiltRing * L::P_BYTES + (k & 1) * L::S_BYTES); };
  const int z0 = ((run * 6 + face) * g.nf + s) * nr;
  const int xP = IOFF + i0 - 4, yP = JOFF + j0 - 3;
  auto issue = [&](int k) {
    uint64_t* b = &bars[k % kFiltRing];
    mbar_expect_tx(b, L::PB * sizeof(T));
    tma_load_3d(smem + (k % kFiltRing) * L::P_BYTES, &a.mP, xP, yP, z0 + k, b);
  };
  if (tid == 0) {
    for (int q = 0; q < kFiltRing; ++q) mbar_init(&bars[q], 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (tid == 0)
    for (int k = 0; k < min(kFiltRing, nr); ++k) issue(k);
  T* out = a.qout + g.vol(run, face, s);
  const long long own = g.at(0, j, i);
  const T f0 = Coef<T>::filt(0), f1 = Coef<T>::filt(1), f2 = Coef<T>::filt(2), f3 = Coef<T>::filt(3);
  T tq[11];
#pragma unroll
  for (int m = 0; m < 11; ++m) tq[m] = T(0);
  bool ok = true;
  for (int k = 0; k < nr; ++k) {
    ok &= mbar_wait(&bars[k % kFiltRing], (k / kFiltRing) & 1, a.err, 3);
    const T* bx = box(k);
    T* t1 = st(k);
    for (int r = ty; r < TY + 6; r += TY) {
      const int jr = j0 - 3 + r;
      const T* row = bx + r * PW + tx + 4;
      T v;
      if (jr < 0 || jr >= n) v = row[0];
      else v = f0 * row[0] + f1 * (row[-1] + row[1]) + f2 * (row[-2] + row[2]) + f3 * (row[-3] + row[3]);
      t1[r * TX + tx] = v;
    }
    if (__syncthreads_or(!ok)) break;
    if (tid == 0 && k + kFiltRing < nr) issue(k + kFiltRing);
    const T* c = t1 + (ty + 3) * TX + tx;
    const T t2 = f0 * c[0] + f1 * (c[-TX] + c[TX]) + f2 * (c[-2 * TX] + c[2 * TX]) + f3 * (c[-3 * TX] + c[3 * TX]);
#pragma unroll
    for (int m = 0; m < 10; ++m) tq[m] = tq[m + 1];
    tq[10] = t2;
    if (k >= 10) {
      T v = Coef<T>::filtr(0) * tq[5];
#pragma unroll
      for (int m = 1; m <= 5; ++m) v += Coef<T>::filtr(m) * (tq[5 - m] + tq[5 + m]);
      out[(long long)(k - 5) * g.plane + own] = v;
    }
    if (k < 5 || k >= nr - 5) out[(long long)k * g.plane + own] = T(0);
  }
  if (!ok && tid == 0)
    for (int q = 0; q < 1000; ++q) __nanosleep(1000);
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
