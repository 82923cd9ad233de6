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
//   adj_stage  mu, the BC mask, the pointwise terms, the sponge, lw and g, and the
//              transposed derivatives of the coefficient-weighted fields: -D_xi and -D_eta
//              with zero halos (the DRP stencil is antisymmetric) and the banded radial
//              transpose, on the interior and on the ghost frame -- the frame values are the
//              adjoints of the neighbour faces' ghost values;
//   adj_rbdy   the one-sided (Tam-Dong) rows of the radial transpose;
//   adj_edge   the transpose of the edge exchange: each source-line point gathers the ghost
//              adjoints that used it, with the same folded coefficients.
// FILTER_EXP^T is the radial transpose, then eta, then xi, each with its ghost-frame
// adjoints, then the same scatter.
#pragma once

#include "kernels.cuh"

namespace solar {

// Fused transposed stage (pointwise part + transposed stencils in one pass).  A CTA owns a
// TX x TY column tile of one face and marches the planes of its chunk (plus three planes on
// either side for the radial window).  Planes stream in through TMA tile loads into a ring of
// shared-memory slots, each guarded by an mbarrier: for a plane of the chunk, the lambda_q
// and lambda_w boxes (tile plus a 4-column / 3-row halo) of v_xi, v_eta, p and rho and the
// tiles of v_r; for the three extra planes on either side only the tiles of p, rho and v_r.
// Every plane also brings its c^2 box (the halo points use it too), the stored divergence
// tile (chunk planes) and its row of radial coefficients (an untiled bulk copy), so the
// per-plane values need no global loads.  Per plane the kernel forms the coefficient-weighted volumes X1, X2 (on the tile and its
// xi halo) and Y1, Y2 (tile and eta halo) in shared memory from mu = lw + beta lq (zero
// outside the face and on the BC planes), applies -D_xi / -D_eta, and keeps facr * R1 and
// facr * R2 of the last seven planes in registers for the banded part of the radial
// transpose, which completes plane k three iterations later.  The rows of the one-sided
// radial stencil (planes 1, 2, nr-3, nr-2; planes 0 and nr-1 carry zero) are written to
// `rb` and added by adj_rbdy_kernel.  Edge tiles also write the ghost-frame adjoints.
// Inputs (lq, lw) and outputs (lout, lwout) are distinct buffers: neighbouring CTAs read the
// inputs' halos.
template <typename T>
struct AdjStageArgs {
  CUtensorMap mBq, mBw;   // boxes (TX+8) x (TY+6) of lq / lw
  CUtensorMap mTq, mTw;   // tiles TX x TY of lq / lw
  CUtensorMap mC2;        // boxes (TX+8) x (TY+6) of the compact c^2 (when present; zero outside the face)
  CUtensorMap mDiv;       // tiles TX x TY of the compact stored divergence (when present)
  T* lout;
  T* lwout;
  T* rb;              // [face][4][2][n*n] raw R1, R2 of planes 1, 2, nr-3, nr-2
  const T* div;       // compact stage-input divergence, or nullptr
  const T* c2;
  double* grad;
  const T* rad;
  const T* met;
  const T* radT;      // [nr][16]: the radial rows of a plane together (through the ring)
  WaitCtl wc;         // error word and bound of the ring waits
  Geom g;
  T alpha, beta, dt, inv_dxi;
  int keep, kchunk;
};

// Ring slots: two in both precisions.  In float that leaves room for three CTAs per SM
// (80 registers, 54 KB of shared memory each): reverse sweep at 6 x 96^3 4.4% faster than
// three slots with two CTAs; four CTAs (64 registers, a 16-byte spill) gained less (1.1%).
template <typename T> struct AdjRing { static constexpr int value = 2; };

template <typename T, int TX, int TY>
struct AdjLayout {
  static constexpr int PW = TX + 8, PH = TY + 6, PB = PW * PH, OB = TX * TY;
  static constexpr size_t P_BYTES = align128(PB * sizeof(T));
  static constexpr size_t O_BYTES = align128(OB * sizeof(T));
  // a chunk plane: boxes [v_xi, v_eta, p, rho] x [lq, lw], then the v_r tiles [lq, lw];
  // an extra plane: tiles [p, rho, v_r] x [lq, lw] from the slot's start; every plane: the
  // c^2 box (the halo points read it too) and (chunk planes) the stored-divergence tile
  // after it, then the plane's row of radial coefficients (16 values, zero padded)
  static constexpr size_t AUX = 8 * P_BYTES + 2 * O_BYTES;
  static constexpr size_t DIV_OFF = AUX + P_BYTES;
  static constexpr size_t RAD_OFF = DIV_OFF + O_BYTES;
  static constexpr size_t SLOT = align128(RAD_OFF + 16 * sizeof(T));
  static constexpr int RING = AdjRing<T>::value;
  static constexpr size_t BAR = RING * SLOT;
  static constexpr size_t TOTAL = BAR + RING * sizeof(uint64_t);
};

template <typename T, int TX, int TY>
__global__ void __launch_bounds__(TX * TY, sizeof(T) == 4 ? 3 : 2) adj_stage_kernel(const __grid_constant__ AdjStageArgs<T> a) {
  using L = AdjLayout<T, TX, TY>;
  constexpr int XW = TX + 6, YH = TY + 6, PW = L::PW;
  constexpr int NHALO = 6 * TX + 6 * TY;
  static_assert(NHALO <= TX * TY, "one halo point per thread");
  __shared__ T sX1[TY][XW], sX2[TY][XW], sY1[YH][TX], sY2[YH][TX];
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L::BAR);
  const Geom& g = a.g;
  const int n = g.n, nr = g.nr;
  const long long P2 = (long long)n * n;
  const int tiles_x = n / TX;
  const int i0 = (blockIdx.x % tiles_x) * TX, j0 = (blockIdx.x / tiles_x) * TY;
  const int face = blockIdx.z;
  const int kb = blockIdx.y * a.kchunk, ke = min(nr, kb + a.kchunk);
  if (kb >= nr) return;
  const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
  const int i = i0 + tx, j = j0 + ty;
  const int p2 = j * n + i;
  const int sRho = g.slot[kRho], sX = g.slot[kVxi], sY = g.slot[kVeta], sR = g.slot[kVr], sP = g.slot[kP];
  const bool has_rho = sRho >= 0;
  const T* __restrict__ met = a.met;
  const T c1 = Coef<T>::drp(1), c2c = Coef<T>::drp(2), c3 = Coef<T>::drp(3);
  // this thread's halo point: eta-halo rows first, then xi-halo columns
  const bool has_halo = tid < NHALO;
  bool xi_halo = false;
  int hi = 0, hj = 0;
  if (tid < 6 * TX) { hi = tid % TX; const int r = tid / TX; hj = r < 3 ? r - 3 : TY + r - 3; }
  else if (has_halo) { xi_halo = true; const int q = tid - 6 * TX; hj = q % TY; const int cc = q / TY; hi = cc < 3 ? cc - 3 : TX + cc - 3; }
  const int hgi = i0 + hi, hgj = j0 + hj;
  const bool h_in = has_halo && hgi >= 0 && hgi < n && hgj >= 0 && hgj < n;
  const int hq2 = h_in ? hgj * n + hgi : 0;
  // 32-bit offsets inside one field volume; the field bases of this face are formed once
  T* const lo_face = a.lout + g.vol(0, face, 0);
  T* const lw_face = a.lwout + g.vol(0, face, 0);
  const int vs = (int)g.vs, plane = (int)g.plane;
  auto fo = [&](int s) { return s * vs; };                          // field base (elements)
  const int own0 = (JOFF + j) * g.pitch + IOFF + i;                 // own point in plane 0
  const int face_c2 = face * nr;                                    // plane index base, compact arrays
  // planes loaded through the ring: every real plane of [kb-3, ke+2]
  const int m_lo = max(kb - 3, 0), m_hi = min(ke + 2, nr - 1);
  const int zf = face * g.nf;            // plane index of (slot s, k) = (zf + s) * nr + k (run 0)
  const int xB = IOFF + i0 - 4, yB = JOFF + j0 - 3, xT = IOFF + i0, yT = JOFF + j0;
  auto slot_base = [&](int sl) { return smem + (size_t)sl * L::SLOT; };
  const bool tc2 = a.c2 != nullptr, tdiv = a.grad != nullptr;   // c^2 / divergence tiles in the ring
  const int zc = face * nr;                // plane index of the compact arrays: face * nr + k
  auto issue = [&](int m, int sl) {
    uint64_t* bar = &bars[sl];
    unsigned char* base = slot_base(sl);
    const bool chunk = m >= kb && m < ke;
    if (tc2) tma_load_3d(base + L::AUX, &a.mC2, i0 - 4, j0 - 3, zc + m, bar);
    if (tdiv && chunk) tma_load_3d(base + L::DIV_OFF, &a.mDiv, i0, j0, zc + m, bar);
    bulk_load(base + L::RAD_OFF, a.radT + (size_t)m * 16, 16 * sizeof(T), bar);
    const uint32_t aux = (uint32_t)(((tc2 ? L::PB : 0) + (tdiv && chunk ? L::OB : 0) + 16) * sizeof(T));
    if (chunk) {
      const int nbox = has_rho ? 4 : 3;
      mbar_expect_tx(bar, (uint32_t)((2 * nbox * L::PB + 2 * L::OB) * sizeof(T)) + aux);
      const int bs[4] = {sX, sY, sP, sRho};
      for (int f = 0; f < nbox; ++f) {
        tma_load_3d(base + (2 * f) * L::P_BYTES, &a.mBq, xB, yB, (zf + bs[f]) * nr + m, bar);
        tma_load_3d(base + (2 * f + 1) * L::P_BYTES, &a.mBw, xB, yB, (zf + bs[f]) * nr + m, bar);
      }
      tma_load_3d(base + 8 * L::P_BYTES, &a.mTq, xT, yT, (zf + sR) * nr + m, bar);
      tma_load_3d(base + 8 * L::P_BYTES + L::O_BYTES, &a.mTw, xT, yT, (zf + sR) * nr + m, bar);
    } else {
      const int nt = has_rho ? 3 : 2;
      mbar_expect_tx(bar, (uint32_t)(2 * nt * L::OB * sizeof(T)) + aux);
      const int ts[3] = {sP, sR, sRho};
      for (int f = 0; f < nt; ++f) {
        tma_load_3d(base + (2 * f) * L::O_BYTES, &a.mTq, xT, yT, (zf + ts[f]) * nr + m, bar);
        tma_load_3d(base + (2 * f + 1) * L::O_BYTES, &a.mTw, xT, yT, (zf + ts[f]) * nr + m, bar);
      }
    }
  };
  if (tid == 0) {
    for (int q = 0; q < L::RING; ++q) mbar_init(&bars[q], 1);
    mbar_fence_init();
  }
  __syncthreads();
  // planes [m_lo, m_issued) have loads issued; thread 0 has seen planes [m_lo, m_seen) land
  int m_issued = m_lo, m_seen = m_lo;
  const bool loads = !a.wc.no_loads;
  if (tid == 0 && loads) {
    tma_prefetch_desc(&a.mBq);
    tma_prefetch_desc(&a.mBw);
    for (int q = 0; q < L::RING && m_issued <= m_hi; ++q, ++m_issued) issue(m_issued, q);
  }
  T w1[7], w2[7];          // facr * R1, facr * R2 of planes m-6 .. m (banded rows only)
  T pp[4], pv[4];          // partial outputs of p and v_r, planes m-3 .. m
#pragma unroll
  for (int q = 0; q < 7; ++q) { w1[q] = T(0); w2[q] = T(0); }
#pragma unroll
  for (int q = 0; q < 4; ++q) { pp[q] = T(0); pv[q] = T(0); }
  // The 2-D metric terms of the own point and of the halo point are the same on every plane
  // and are held in registers for the whole chunk (the per-plane reads were the kernel's
  // main long-scoreboard stall).  In double this spills 28 bytes under the 128-register
  // budget and still ran 1% faster than four 16-byte reads per plane.
  const T gD = __ldg(met + mD * P2 + p2), gXYD = __ldg(met + mXYD * P2 + p2);
  const T gC = __ldg(met + mC * P2 + p2), gXYC = __ldg(met + mXYC * P2 + p2);
  const T gDivX = __ldg(met + mDivX * P2 + p2), gDivY = __ldg(met + mDivY * P2 + p2);
  const T gTX = __ldg(met + mTX * P2 + p2), gTY = __ldg(met + mTY * P2 + p2);
  T gh1 = T(0), gh2 = T(0), gh3 = T(0);
  if (h_in) {
    gh1 = __ldg(met + (xi_halo ? mD : mXYD) * P2 + hq2);
    gh2 = __ldg(met + (xi_halo ? mXYC : mC) * P2 + hq2);
    gh3 = __ldg(met + (xi_halo ? mDivX : mDivY) * P2 + hq2);
  }
  int slot = 0;
  uint32_t phase = 0;
  bool ok = true, failed = false;
  const int bo = (ty + 3) * PW + tx + 4;           // own point in a box
  const int to = ty * TX + tx;                     // own point in a tile
  for (int m = kb - 3; m <= ke + 2; ++m) {
    const bool real = (m >= 0 && m < nr);
    const bool own = (m >= kb && m < ke);
    const bool bc = (m == 0 || m == nr - 1);
    T r1 = T(0), r2 = T(0), part_p = T(0), part_v = T(0), facr_m = T(0);
    if (real) {
      const int o = m * plane + own0;
      const long long plane_c2 = (long long)(face_c2 + m) * P2;
      const bool do_halo = own && h_in && !bc;
      // the gradient accumulator is read before the ring wait, so that its DRAM latency
      // passes during the wait and the plane's arithmetic instead of stalling the store
      const double gacc = (own && a.grad) ? a.grad[plane_c2 + p2] : 0.0;
      if (ok) {
        ok = mbar_wait(&bars[slot], phase, a.wc, kErrAdjointRing);
        if (ok) m_seen = m + 1;
      }
      const T* sb = reinterpret_cast<const T*>(slot_base(slot));
      const T* rrow = reinterpret_cast<const T*>(slot_base(slot) + L::RAD_OFF);
      const T invr = rrow[rInvR], inv_rho0 = rrow[rInvRho0], rho0 = rrow[rRho0], c2r = rrow[rC2Rho0];
      facr_m = rrow[rFacR];
      constexpr int PBs = (int)(L::P_BYTES / sizeof(T)), OBs = (int)(L::O_BYTES / sizeof(T));
      const T* sc2 = reinterpret_cast<const T*>(slot_base(slot) + L::AUX);
      const T c2own = tc2 ? sc2[bo] : T(0);
      const T divv = (own && tdiv) ? sc2[(L::DIV_OFF - L::AUX) / sizeof(T) + to] : T(0);
      T lqv[5], lwv[5];
#pragma unroll
      for (int f = 0; f < 5; ++f) { lqv[f] = T(0); lwv[f] = T(0); }
      if (own) {
        const int bf[4] = {kVxi, kVeta, kP, kRho};
#pragma unroll
        for (int f = 0; f < 4; ++f) {
          if (f == 3 && !has_rho) continue;
          lqv[bf[f]] = sb[(2 * f) * PBs + bo];
          lwv[bf[f]] = sb[(2 * f + 1) * PBs + bo];
        }
        lqv[kVr] = sb[8 * PBs + to];
        lwv[kVr] = sb[8 * PBs + OBs + to];
      } else {
        lqv[kP] = sb[to];
        lwv[kP] = sb[OBs + to];
        lqv[kVr] = sb[2 * OBs + to];
        lwv[kVr] = sb[3 * OBs + to];
        if (has_rho) { lqv[kRho] = sb[4 * OBs + to]; lwv[kRho] = sb[5 * OBs + to]; }
      }
      T mu[5], mp[5];
#pragma unroll
      for (int f = 0; f < 5; ++f) {
        mu[f] = lwv[f] + a.beta * lqv[f];
        mp[f] = bc ? T(0) : mu[f];
      }
      const T c2rho0 = a.c2 ? c2own * rho0 : c2r;
      const T e = -c2rho0 * mp[kP] - rho0 * mp[kRho];
      r1 = -inv_rho0 * mp[kVr];
      r2 = e;
      if (own) {
        sX1[ty][tx + 3] = -invr * inv_rho0 * (gD * mp[kVxi] + gXYC * mp[kVeta]);
        sX2[ty][tx + 3] = invr * gDivX * e;
        sY1[ty + 3][tx] = -invr * inv_rho0 * (gXYD * mp[kVxi] + gC * mp[kVeta]);
        sY2[ty + 3][tx] = invr * gDivY * e;
        if (has_halo) {
          T v1 = T(0), v2 = T(0);
          if (do_halo) {
            const int hb = (hj + 3) * PW + hi + 4;
            const T hx = sb[1 * PBs + hb] + a.beta * sb[0 * PBs + hb];
            const T hy = sb[3 * PBs + hb] + a.beta * sb[2 * PBs + hb];
            const T hp = sb[5 * PBs + hb] + a.beta * sb[4 * PBs + hb];
            const T hr = has_rho ? sb[7 * PBs + hb] + a.beta * sb[6 * PBs + hb] : T(0);
            const T he = -(a.c2 ? sc2[hb] * rho0 : c2r) * hp - rho0 * hr;
            v1 = -invr * inv_rho0 * (gh1 * hx + gh2 * hy);
            v2 = invr * gh3 * he;
          }
          if (xi_halo) { sX1[hj][hi + 3] = v1; sX2[hj][hi + 3] = v2; }
          else { sY1[hj + 3][hi] = v1; sY2[hj + 3][hi] = v2; }
        }
        // pointwise terms, lw update, gradient
        const T sig = rrow[rSigma];
        T pw[5];
        pw[kRho] = -rrow[rG0Rho0] * mp[kVr] - sig * mu[kRho];
        pw[kVxi] = -invr * gTX * e;
        pw[kVeta] = -invr * gTY * e;
        pw[kVr] = T(2) * invr * e - rrow[rDRho0] * mp[kRho] + rrow[rRho0G0] * mp[kP] - sig * mu[kVr];
        pw[kP] = -sig * mu[kP];
#pragma unroll
        for (int f = 0; f < 5; ++f) {
          const int s = g.slot[f];
          if (s < 0) continue;
          lw_face[fo(s) + o] = a.alpha * mu[f];
          const T base = (a.keep ? lqv[f] : T(0)) + a.dt * pw[f];
          if (f == kP) part_p = base;
          else if (f == kVr) part_v = base;
          else if (f == kRho) lo_face[fo(s) + o] = base;
          else lqv[f] = base;                                  // v_xi, v_eta: 2-D part added below
        }
        if (a.grad) {
          const T c = sqrt(c2rho0 * inv_rho0);
          a.grad[plane_c2 + p2] = gacc + (double)(a.dt * (T(-2) * c * rho0 * divv) * mp[kP]);
        }
        if (m == 1 || m == 2 || m == nr - 3 || m == nr - 2) {
          const int row = m <= 2 ? m - 1 : m - (nr - 3) + 2;
          T* rbp = a.rb + (((long long)face * 4 + row) * 2) * P2 + p2;
          rbp[0] = r1;
          rbp[P2] = r2;
        }
        __syncthreads();
        const T* x1 = &sX1[ty][tx + 3];
        const T* x2 = &sX2[ty][tx + 3];
        const T* y1 = &sY1[ty + 3][tx];
        const T* y2 = &sY2[ty + 3][tx];
        const T dx1 = c1 * (x1[1] - x1[-1]) + c2c * (x1[2] - x1[-2]) + c3 * (x1[3] - x1[-3]);
        const T dx2 = c1 * (x2[1] - x2[-1]) + c2c * (x2[2] - x2[-2]) + c3 * (x2[3] - x2[-3]);
        const T dy1 = c1 * (y1[TX] - y1[-TX]) + c2c * (y1[2 * TX] - y1[-2 * TX]) + c3 * (y1[3 * TX] - y1[-3 * TX]);
        const T dy2 = c1 * (y2[TX] - y2[-TX]) + c2c * (y2[2 * TX] - y2[-2 * TX]) + c3 * (y2[3 * TX] - y2[-3 * TX]);
        const T k2 = -a.dt * a.inv_dxi;
        part_p += k2 * (dx1 + dy1);
        lo_face[fo(sX) + o] = lqv[kVxi] + k2 * dx2;
        lo_face[fo(sY) + o] = lqv[kVeta] + k2 * dy2;
        // ghost-frame adjoints of the neighbour faces' values (W/E columns, S/N rows)
        if ((i0 == 0 && tx < 3) || (i0 + TX == n && tx >= TX - 3)) {
          const bool west = i0 == 0 && tx < 3;
          const int c = west ? tx : TX + 3 + (tx - (TX - 3));  // x index of the ghost column
          auto xv = [&](const T* row, int q) { return (q >= 0 && q < XW) ? row[q] : T(0); };
          const T* r1p = &sX1[ty][0];
          const T* r2p = &sX2[ty][0];
          const T f1 = c1 * (xv(r1p, c + 1) - xv(r1p, c - 1)) + c2c * (xv(r1p, c + 2) - xv(r1p, c - 2)) + c3 * (xv(r1p, c + 3) - xv(r1p, c - 3));
          const T f2 = c1 * (xv(r2p, c + 1) - xv(r2p, c - 1)) + c2c * (xv(r2p, c + 2) - xv(r2p, c - 2)) + c3 * (xv(r2p, c + 3) - xv(r2p, c - 3));
          const int og = o - i + (west ? tx - 3 : n + (tx - (TX - 3)));
          lo_face[fo(sP) + og] = k2 * f1;
          lo_face[fo(sX) + og] = k2 * f2;
        }
        if ((j0 == 0 && ty < 3) || (j0 + TY == n && ty >= TY - 3)) {
          const bool south = j0 == 0 && ty < 3;
          const int r = south ? ty : TY + 3 + (ty - (TY - 3));  // y index of the ghost row
          auto yv = [&](const T (*col)[TX], int q) { return (q >= 0 && q < YH) ? col[q][tx] : T(0); };
          const T f1 = c1 * (yv(sY1, r + 1) - yv(sY1, r - 1)) + c2c * (yv(sY1, r + 2) - yv(sY1, r - 2)) + c3 * (yv(sY1, r + 3) - yv(sY1, r - 3));
          const T f2 = c1 * (yv(sY2, r + 1) - yv(sY2, r - 1)) + c2c * (yv(sY2, r + 2) - yv(sY2, r - 2)) + c3 * (yv(sY2, r + 3) - yv(sY2, r - 3));
          const int og = o + ((south ? ty - 3 : n + (ty - (TY - 3))) - j) * g.pitch;
          lo_face[fo(sP) + og] = k2 * f1;
          lo_face[fo(sY) + og] = k2 * f2;
        }
      }
    }
    // radial windows and the partial-output ring advance one plane
    const bool band = real && m >= 3 && m <= nr - 4;
    const T facr = band ? facr_m : T(0);
#pragma unroll
    for (int q = 0; q < 6; ++q) { w1[q] = w1[q + 1]; w2[q] = w2[q + 1]; }
    w1[6] = facr * r1;
    w2[6] = facr * r2;
#pragma unroll
    for (int q = 0; q < 3; ++q) { pp[q] = pp[q + 1]; pv[q] = pv[q + 1]; }
    pp[3] = part_p;
    pv[3] = part_v;
    const int pl = m - 3;
    if (pl >= kb && pl < ke) {
      // (Dr^T R)_pl = sum_d a_d facr_{pl-d} R_{pl-d}, a_{-d} = -a_d; window index of pl-d is 3-d
      const T rp = c1 * (w1[2] - w1[4]) + c2c * (w1[1] - w1[5]) + c3 * (w1[0] - w1[6]);
      const T rv = c1 * (w2[2] - w2[4]) + c2c * (w2[1] - w2[5]) + c3 * (w2[0] - w2[6]);
      const int op = pl * plane + own0;
      lo_face[fo(sP) + op] = pp[0] + a.dt * rp;
      lo_face[fo(sR) + op] = pv[0] + a.dt * rv;
    }
    if (real) {
      // every thread is done with this slot (and with the X/Y arrays): refill it
      if (__syncthreads_or(!ok)) { failed = true; break; }
      if (tid == 0 && loads && m_issued <= m_hi) issue(m_issued++, slot);
      if (++slot == L::RING) { slot = 0; phase ^= 1; }
    }
  }
  // a wait gave up: wait (bounded) for the loads still in flight before the CTA exits
  if (failed && tid == 0) mbar_drain(bars, L::RING, m_lo, m_seen, m_issued, a.wc.polls);
}

// The one-sided radial rows 1, 2 (onto planes 0..6) and nr-3, nr-2 (onto planes nr-7..nr-1)
// of the radial transpose, added to p and v_r after adj_stage_kernel.
template <typename T>
__global__ void adj_rbdy_kernel(T* lout, const T* rb, const T* rad, Geom g, T dt) {
  const int n = g.n, nr = g.nr;
  const long long P2 = (long long)n * n;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= 6 * 14 * P2) return;
  const int face = (int)(idx / (14 * P2));
  const int q = (int)((idx / P2) % 14);
  const int p2 = (int)(idx % P2), i = p2 % n, j = p2 / n;
  const bool low = q < 7;
  const int pl = low ? q : nr - 14 + q;                      // planes 0..6 or nr-7..nr-1
  T s1 = T(0), s2 = T(0);
  for (int r = 0; r < 2; ++r) {
    const int kk = low ? 1 + r : nr - 3 + r;
    const int row = low ? r : 2 + r;
    const T* rbp = rb + (((long long)face * 4 + row) * 2) * P2 + p2;
    const T f = rad[rFacR * nr + kk];
    const T b = low ? Coef<T>::bdy(kk, pl) : -Coef<T>::bdy(nr - 1 - kk, nr - 1 - pl);
    s1 += f * b * rbp[0];
    s2 += f * b * rbp[P2];
  }
  const long long o = g.at(pl, j, i);
  lout[g.vol(0, face, g.slot[kP]) + o] += dt * s1;
  lout[g.vol(0, face, g.slot[kVr]) + o] += dt * s2;
}

// Transpose of the edge exchange, as a gather: every source-line point (the receiving face
// and edge's route, layer l, position u along the source edge, plane k) sums the ghost
// adjoints of the ghost points whose 9 taps include it -- a contiguous range of positions t,
// tspan -- then adds the sum to its value (atomically: the source lines of two edges of a
// face share their corner points).  The CTA first copies the ghost values its positions
// need (the union of their ranges, one read per ghost point and field) into shared memory:
// on W/E receivers those are column entries, one scattered request each.  The weights come
// from a table transposed on the host, wt[kind][row][j][u] = the folded coefficient with
// which ghost point t = lo(u) + j of row (face-edge, layer) used source position u (kind 0
// scalar, 1 and 2 the vector pair), read contiguously across u.  mode 0: p scalar + the
// rotated vector component (v_xi on W/E receivers, v_eta on S/N); mode 1: every stored
// field scalar.  grid: x over u, y over (receiving face-edge, layer), z over planes; dynamic
// shared memory: (mode 0 ? 2 : nf) x n values.
template <typename T>
__global__ void adj_edge_kernel(T* q, const T* __restrict__ wt, int span, const int* __restrict__ tspan, Geom g,
                                int mode) {
  extern __shared__ __align__(16) unsigned char aesm[];
  T* const sg = reinterpret_cast<T*>(aesm);               // [field][t]
  __shared__ int s_lo, s_hi;
  const int n = g.n;
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  const int fe = blockIdx.y / 3, l = blockIdx.y % 3, k = blockIdx.z;
  const int face = fe >> 2, e = fe & 3;
  const EdgeRouteDev rt = cRoute[face][e];
  const bool along_i = rt.src_edge <= 1;
  const int fixed = (rt.src_edge == 0 || rt.src_edge == 2) ? l + 1 : n - 2 - l;
  const int row = fe * 3 + l;
  int lo = 0, hi = -1;
  if (u < n) {
    lo = __ldg(tspan + (row * n + u) * 2);
    hi = __ldg(tspan + (row * n + u) * 2 + 1);
  }
  if (threadIdx.x == 0) { s_lo = n; s_hi = -1; }
  __syncthreads();
  if (hi >= lo) { atomicMin(&s_lo, lo); atomicMax(&s_hi, hi); }
  __syncthreads();
  const int tmin = s_lo, tmax = s_hi;
  if (tmax < tmin) return;                                 // no ghost point uses this block
  // receiver ghost position of (e, l, t): rows -1-l / n+l, columns -1-l / n+l
  const long long g0 = (e == 0) ? g.at(k, -1 - l, 0) : (e == 1) ? g.at(k, n + l, 0)
                     : (e == 2) ? g.at(k, 0, -1 - l) : g.at(k, 0, n + l);
  const long long gstep = e <= 1 ? 1 : g.pitch;
  const int nfs = mode == 1 ? g.nf : 2;
  auto slot_of = [&](int f) {
    return mode == 1 ? f : (f == 0 ? g.slot[kP] : (e >= 2 ? g.slot[kVxi] : g.slot[kVeta]));
  };
  for (int f = 0; f < nfs; ++f) {
    const T* gv = q + g.vol(0, face, slot_of(f)) + g0;
    for (int t = tmin + threadIdx.x; t <= tmax; t += blockDim.x) sg[f * n + t] = gv[t * gstep];
  }
  __syncthreads();
  if (hi < lo) return;
  const long long src = g.at(k, along_i ? fixed : u, along_i ? u : fixed);
  const long long kind = 72LL * span * n;                 // stride between weight kinds
  const T* w = wt + (long long)row * span * n + u;        // weight of ghost lo + j at w[j * n]
  const int cnt = hi - lo + 1;
  if (mode == 1) {
    for (int f = 0; f < nfs; ++f) {
      const T* gs = sg + f * n + lo;
      T acc = T(0);
      for (int j = 0; j < cnt; ++j) acc += __ldg(w + j * n) * gs[j];
      atomicAdd(q + g.vol(0, rt.src_face, f) + src, acc);
    }
    return;
  }
  const T* gp = sg + lo;
  const T* gvv = sg + n + lo;
  T ap = T(0), ax = T(0), ay = T(0);
  for (int j = 0; j < cnt; ++j) {
    const T pv = gp[j], vv = gvv[j];
    ap += __ldg(w + j * n) * pv;
    ax += __ldg(w + kind + j * n) * vv;
    ay += __ldg(w + 2 * kind + j * n) * vv;
  }
  atomicAdd(q + g.vol(0, rt.src_face, g.slot[kP]) + src, ap);
  atomicAdd(q + g.vol(0, rt.src_face, g.slot[kVxi]) + src, ax);
  atomicAdd(q + g.vol(0, rt.src_face, g.slot[kVeta]) + src, ay);
}

// FILTER_R^T for every stored field: u_m = sum over output planes k in [5, nr-6] of
// fr_{|k-m|} lam_k (the end planes of the forward output are constant zeros).  One thread
// per (field volume, j, i) column marches the planes with an 11-deep register queue, so
// lam is read once.
template <typename T>
__global__ void adj_filter_r_kernel(const T* lam, T* u, Geom g) {
  const int n = g.n, nr = g.nr;
  const long long P = (long long)n * n;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)g.nruns * 6 * g.nf * P) return;
  const long long vsel = idx / P;                      // (run*6 + face)*nf + slot
  const int p2 = (int)(idx % P), i = p2 % n, j = p2 / n;
  const T* L = lam + vsel * g.vs + g.at(0, j, i);
  T* U = u + vsel * g.vs + g.at(0, j, i);
  auto ld = [&](int k) { return (k >= 5 && k <= nr - 6) ? L[(long long)k * g.plane] : T(0); };
  T q[11];
#pragma unroll
  for (int d = 0; d < 11; ++d) q[d] = ld(d - 5);     // planes m-5 .. m+5 for m = 0
  for (int m = 0; m < nr; ++m) {
    T s = Coef<T>::filtr(0) * q[5];
#pragma unroll
    for (int d = 1; d <= 5; ++d) s += Coef<T>::filtr(d) * (q[5 - d] + q[5 + d]);
    U[(long long)m * g.plane] = s;
#pragma unroll
    for (int d = 0; d < 10; ++d) q[d] = q[d + 1];
    q[10] = ld(m + 6);
  }
}

// FILTER_XI^T (FILTER_ETA^T (u)) for one TX x TY tile of one field volume, plane by plane:
// the transposes of the two in-face filters of FILTER_EXP with zero halos.  u (the adjoint
// of the eta filter's output) lives on the face interior only.  Each thread owns V consecutive points
// (V = 16 bytes / sizeof(T)) of one tile row.  Per plane: the box of u (tile rows +-3, tile
// columns -4 .. +3, zero outside the face) goes to shared memory; every thread eta-filters
// its row over the box's vector columns (the first two thread columns also take the two
// halo vectors); threads next to an S/N face edge write the eta filter's halo adjoints
// (v on the ghost rows, the unfiltered-halo part) to the frame; after a barrier each thread
// xi-filters its V points from NV vectors of v, and the threads at a W/E face edge write
// the xi filter's halo adjoints to the ghost columns.  u and v are double-buffered, so a
// plane costs two barriers.  (A scalar form with one point per thread and three barriers per
// plane took 136 us in float and 214 us in double per launch at 6 x 96^3; the reverse sweep
// of 200 steps 252 -> 239 ms in float, 435 -> 427 ms in double.)
template <typename T, int TX, int TY>
__global__ void __launch_bounds__((TX / Vec16<T>::V) * TY) adj_filter_xyv_kernel(const T* __restrict__ in, T* out,
                                                                                Geom g, int kp) {
  constexpr int V = Vec16<T>::V, NT = TX / V, NTH = NT * TY;
  constexpr int BW = TX + 8, BH = TY + 6, NG = BW / V;       // box: columns i0-4 .. i0+TX+3
  constexpr int NBV = BH * NG, PER = (NBV + NTH - 1) / NTH;
  constexpr int NV = (V + 8) / V;                            // vectors covering columns c-4 .. c+V+3
  constexpr int Q0 = 4 / V;                                  // box vector of tile column 0
  __shared__ __align__(16) T su[2][BH][BW];
  __shared__ __align__(16) T sv[2][TY][BW];
  const int n = g.n, tiles_x = n / TX;
  const int i0 = (blockIdx.x % tiles_x) * TX, j0 = (blockIdx.x / tiles_x) * TY;
  const int k0 = blockIdx.y * kp, k1 = min(g.nr, k0 + kp);
  const long long vbase = (long long)blockIdx.z * g.vs;
  const int cx = threadIdx.x, ty = threadIdx.y, tid = ty * NT + cx;
  const T f0 = Coef<T>::filt(0), f1 = Coef<T>::filt(1), f2 = Coef<T>::filt(2), f3 = Coef<T>::filt(3);
  int boff[PER];
#pragma unroll
  for (int e = 0; e < PER; ++e) {
    const int q = tid + e * NTH;
    const int br = q / NG, bq = q % NG;
    const int gj = j0 - 3 + br, gi = i0 - 4 + V * bq;
    boff[e] = (q < NBV && gj >= 0 && gj < n && gi >= 0 && gi < n) ? (JOFF + gj) * g.pitch + IOFF + gi : -1;
  }
  T nxt[PER][V];
  auto fetch = [&](int k) {
    const T* u = in + vbase + (long long)k * g.plane;
#pragma unroll
    for (int e = 0; e < PER; ++e) {
      if (boff[e] >= 0) {
        ldv(u + boff[e], nxt[e]);
      } else {
#pragma unroll
        for (int c = 0; c < V; ++c) nxt[e][c] = T(0);
      }
    }
  };
  if (k0 < k1) fetch(k0);
  for (int k = k0; k < k1; ++k) {
    const int b = k & 1;
#pragma unroll
    for (int e = 0; e < PER; ++e) {
      const int q = tid + e * NTH;
      if (q < NBV) stv(&su[b][q / NG][(q % NG) * V], nxt[e]);
    }
    __syncthreads();
    if (k + 1 < k1) fetch(k + 1);
    // eta^T on the tile rows, every vector column of the box
    for (int q = cx; q < NG; q += NT) {
      T c[7][V];
#pragma unroll
      for (int m = 0; m < 7; ++m) ldv(&su[b][ty + m][q * V], c[m]);
      T v[V];
#pragma unroll
      for (int e = 0; e < V; ++e)
        v[e] = f0 * c[3][e] + f1 * (c[2][e] + c[4][e]) + f2 * (c[1][e] + c[5][e]) + f3 * (c[0][e] + c[6][e]);
      stv(&sv[b][ty][q * V], v);
    }
    T* o = out + vbase + (long long)k * g.plane;
    // eta-filter halo adjoints: v on the ghost rows (box rows 0..2 / TY+3..TY+5), tile columns
    for (int side = 0; side < 2; ++side) {
      const bool edge = side == 0 ? (j0 == 0 && ty < 3) : (j0 + TY == n && ty >= TY - 3);
      if (!edge) continue;
      const int r = side == 0 ? ty : ty + 6;                 // box row
      T v[V];
#pragma unroll
      for (int e = 0; e < V; ++e) v[e] = T(0);
      auto U = [&](int br, int e) { return (br >= 0 && br < BH) ? su[b][br][(Q0 + cx) * V + e] : T(0); };
#pragma unroll
      for (int e = 0; e < V; ++e)
        v[e] = f0 * U(r, e) + f1 * (U(r - 1, e) + U(r + 1, e)) + f2 * (U(r - 2, e) + U(r + 2, e)) +
               f3 * (U(r - 3, e) + U(r + 3, e));
      stv(o + (JOFF + j0 - 3 + r) * g.pitch + IOFF + i0 + V * cx, v);
    }
    __syncthreads();
    // xi^T on the tile: w holds box columns V*cx .. V*cx + NV*V - 1; the own point e sits at
    // box column V*cx + 4 + e
    T w[NV * V];
#pragma unroll
    for (int m = 0; m < NV; ++m) ldv(&sv[b][ty][(cx + m) * V], w + m * V);
    auto W = [&](int idx) { return (idx >= 0 && idx < NV * V) ? w[idx] : T(0); };
    auto xt = [&](int c) {                                   // c = index into w
      return f0 * W(c) + f1 * (W(c - 1) + W(c + 1)) + f2 * (W(c - 2) + W(c + 2)) + f3 * (W(c - 3) + W(c + 3));
    };
    T r[V];
#pragma unroll
    for (int e = 0; e < V; ++e) r[e] = xt(4 + e);
    stv(o + (JOFF + j0 + ty) * g.pitch + IOFF + i0 + V * cx, r);
    // xi-filter halo adjoints on the ghost columns (box columns 1..3 / TX+4..TX+6)
    if (i0 == 0 && cx == 0) {
#pragma unroll
      for (int c = 1; c <= 3; ++c) o[(JOFF + j0 + ty) * g.pitch + IOFF - 4 + c] = xt(c);
    }
    if (i0 + TX == n && cx == NT - 1) {
#pragma unroll
      for (int c = TX + 4; c <= TX + 6; ++c) o[(JOFF + j0 + ty) * g.pitch + IOFF + i0 - 4 + c] = xt(c - V * cx);
    }
  }
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

}  // namespace solar
