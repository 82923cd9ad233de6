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

#include "scheme.h"
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
  int face0, nface;         // zones the step kernels work on (a process owning part of the sphere)
  int k0, k1;               // radial planes the step kernels compute (a process owning a radial slab)
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

__host__ __device__ constexpr size_t align128(size_t b) { return (b + 127) / 128 * 128; }

// 16-byte vectors: V = 4 floats or 2 doubles.
template <typename T> struct Vec16;
template <> struct Vec16<float> { using type = float4; static constexpr int V = 4; };
template <> struct Vec16<double> { using type = double2; static constexpr int V = 2; };

template <typename T>
__device__ __forceinline__ void ldv(const T* p, T* out) {
  using VT = typename Vec16<T>::type;
  const VT v = *reinterpret_cast<const VT*>(p);
  const T* e = reinterpret_cast<const T*>(&v);
#pragma unroll
  for (int q = 0; q < Vec16<T>::V; ++q) out[q] = e[q];
}
template <typename T>
__device__ __forceinline__ void stv(T* p, const T* in) {
  using VT = typename Vec16<T>::type;
  VT v;
  T* e = reinterpret_cast<T*>(&v);
#pragma unroll
  for (int q = 0; q < Vec16<T>::V; ++q) e[q] = in[q];
  *reinterpret_cast<VT*>(p) = v;
}

// One 32-byte sector in a single 256-bit store (sm_100); p must be 32-byte aligned.
__device__ __forceinline__ void st_sector(float* p, const float* v) {
  asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(p), "f"(v[0]), "f"(v[1]), "f"(v[2]),
               "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7])
               : "memory");
}
__device__ __forceinline__ void st_sector(double* p, const double* v) {
  asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(p), "d"(v[0]), "d"(v[1]), "d"(v[2]), "d"(v[3])
               : "memory");
}

// Two floats in one 64-bit register for the paired FP32 arithmetic of sm_100
// (add/mul/fma .f32x2: one instruction for both lanes, each rounded as the scalar one).
__device__ __forceinline__ unsigned long long pk2(float x, float y) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(x), "f"(y));
  return r;
}
__device__ __forceinline__ void upk2(unsigned long long r, float& x, float& y) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(x), "=f"(y) : "l"(r));
}
__device__ __forceinline__ unsigned long long add2(unsigned long long a, unsigned long long b) {
  unsigned long long d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ unsigned long long mul2(unsigned long long a, unsigned long long b) {
  unsigned long long d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ unsigned long long fma2(unsigned long long a, unsigned long long b, unsigned long long c) {
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}

// ---------------------------------------------------------------------------------
// Edge (ghost) kernel: INTERPOLATE_ALONG_X/Y + TRANSFORM_VECTOR_BETWEEN_MESHES_DIV + the
// inter-zone exchange and its reversal, in one pass.  Every ghost value is a 9-tap sum
// over one source line: the scalar weights are the Lagrange weights; the vector
// coefficients fold the Lagrange weight, the source face's (xi,eta)->(theta,phi)
// conversion and the receiver-frame rotation into one pair per tap.
// mode 0: RHS halos -- p scalar on all edges; v_xi on W/E and v_eta on S/N, rotated.
// mode 1: filter halos -- every stored field, scalar, all edges (filter.f90:23-28).
template <typename T>
struct EdgeArgs {
  CUtensorMap mRow;         // tiles {sp, 3 rows} of the buffer (source lines along i)
  CUtensorMap mCol;         // tiles {4, sp rows} of the buffer (source lines along j)
  T* q;                     // buffer whose frames are filled (its interior is the source)
  const T* ew;              // [6][4][3][9][n]     scalar tap weights, position fastest
  const T* eg;              // [6][4][3][9][2][n]  vector tap weights (v_xi, v_eta)
  const int* s0t;           // [6][4][3][n]        first tap along the source edge
  const int* runs;          // stored run of each launched run index (grid z), or nullptr
  const int2* win;          // [24][nseg] staged source window (first position, count)
  Geom g;
  int mode;
  int kchunk;               // planes per CTA
  int ts, nseg;             // positions per segment, segments per edge
  int ngroups;              // field groups per edge: 2 in mode 0, ceil(nf / 2) in mode 1
  int sp;                   // staged positions per line (window capacity, a multiple of 8)
  WaitCtl wc;               // error word and bound of the ring waits
};

// One CTA per (run, receiving face and edge, field group, segment of ts positions along
// the edge, chunk of planes).  Field groups: mode 0 -> {p} and {v_xi, v_eta} (one rotated
// output); mode 1 -> pairs of stored fields, each scalar.  Each of the 3 * ts threads owns
// one (layer, position) ghost point and keeps its 9 (scalar) or 18 (vector) tap weights in
// registers for the whole chunk, while the CTA marches the planes through kEdgeRing staging
// slots that thread 0 fills with TMA tile loads kEdgeDepth planes ahead of the plane being
// computed (one mbarrier per slot):
//   source lines along i (S/N source edges): box {sp, 3 rows} per field -> [row][u];
//   source lines along j (W/E): the three columns of a row lie in one aligned 4-value
//     group; box {4, sp rows} per field -> [u][4], spread to [layer][u] one plane before
//     use (tap reads from the 4-value groups would be 4-way bank conflicts).
// A tile load is one request for the whole strided box, so a plane's 3 x sp source values
// cost the SM no per-row load instructions and no per-row miss tracking.
// S/N receivers store their ghost rows directly.  W/E receivers park a plane's results in
// shared memory and one thread per row writes the row's whole 32-byte sector (ghost
// columns plus the padding next to them): writing 12 of 32 bytes would make the L2 read
// the sector back from DRAM to merge it.
constexpr int kEdgeDepth = 3;               // planes in flight ahead of the computed one
constexpr int kEdgeRing = kEdgeDepth + 2;   // a slot is refilled two planes after its last read

// Shared memory of one CTA in bytes: staging ring (two fields of 4 * sp values per slot),
// spread planes, parked W/E results, one mbarrier per slot.
__host__ __device__ inline int edge_smem_bytes(int sp, int ts, int esize) {
  return (kEdgeRing * 8 * sp + 16 * sp + 12 * ts) * esize + kEdgeRing * 8;
}

// Resident CTAs per SM the registers are budgeted for (3 x 384 threads in float).
template <typename T> struct EdgeMinBlocks { static constexpr int value = sizeof(T) == 4 ? 3 : 2; };

template <typename T>
__global__ void __launch_bounds__(384, (EdgeMinBlocks<T>::value)) edge_kernel(const __grid_constant__ EdgeArgs<T> a) {
  extern __shared__ __align__(128) unsigned char esm[];
  const Geom& g = a.g;
  const int n = g.n, ts = a.ts, sp = a.sp;
  // the run map is written before the launches that use it and constant during them
  const int run = a.runs ? a.runs[blockIdx.z] : blockIdx.z;
  const int kb = g.k0 + blockIdx.x * a.kchunk;
  if (kb >= g.k1) return;
  const int kc = min(a.kchunk, g.k1 - kb);
  int y = blockIdx.y;
  const int seg = y % a.nseg;
  y /= a.nseg;
  const int grp = y % a.ngroups;
  const int fe = g.face0 * 4 + y / a.ngroups, face = fe >> 2, e = fe & 3;
  const EdgeRouteDev rt = cRoute[face][e];
  const bool along_i = rt.src_edge <= 1;                 // S/N source lines run along i
  const bool low = (rt.src_edge == 0 || rt.src_edge == 2);
  const bool cols = e >= 2;                              // W/E receiver: ghost columns
  const bool vec = a.mode != 1 && grp == 1;              // {v_xi, v_eta} -> one rotated component
  int nsrc, nout, sl0, sl1, ol0, ol1;
  if (a.mode == 1) {
    sl0 = ol0 = 2 * grp;
    sl1 = ol1 = min(2 * grp + 1, g.nf - 1);
    nsrc = nout = min(2, g.nf - 2 * grp);
  } else if (!vec) {
    sl0 = sl1 = ol0 = ol1 = g.slot[kP];
    nsrc = nout = 1;
  } else {
    sl0 = g.slot[kVxi];
    sl1 = g.slot[kVeta];
    ol0 = ol1 = cols ? g.slot[kVxi] : g.slot[kVeta];
    nsrc = 2;
    nout = 1;
  }
  const int lo = a.win[fe * a.nseg + seg].x;             // first staged source position
  const int tid = threadIdx.x;
  const int l = tid / ts, tl = tid - l * ts, t = seg * ts + tl;
  const bool valid = t < n;
  constexpr int SECT = 32 / sizeof(T);                   // elements per 32-byte sector
  const int FS = 4 * sp;                                 // field stride inside a slot / spread plane
  const int SLOT = 2 * FS;
  T* const sm = reinterpret_cast<T*>(esm);
  T* const tb = sm + kEdgeRing * SLOT;                   // [2][2 fields][4 sp]: [layer][u] planes
  T* const res = tb + 4 * FS;                            // [2][2 outputs][3 layers][ts]
  uint64_t* const bars = reinterpret_cast<uint64_t*>(res + 12 * ts);

  // tap weights and window offset of this thread's ghost point
  T c0[9], c1[9];
  const int s0 = valid ? a.s0t[((long long)fe * 3 + l) * n + t] - lo : 0;   // idle threads read the window start
  {
    const int tc = valid ? t : 0;
    const long long crow = ((long long)fe * 3 + l) * 9;
#pragma unroll
    for (int s = 0; s < 9; ++s) {
      if (vec) {
        c0[s] = a.eg[((crow + s) * 2 + 0) * n + tc];
        c1[s] = a.eg[((crow + s) * 2 + 1) * n + tc];
      } else {
        c0[s] = a.ew[(crow + s) * n + tc];
        c1[s] = T(0);
      }
    }
  }
  // tile coordinates of the chunk's first plane (z counts planes over run, face, field, k)
  const int zs0 = ((run * 6 + rt.src_face) * g.nf + sl0) * g.nr + kb;
  const int zs1 = ((run * 6 + rt.src_face) * g.nf + sl1) * g.nr + kb;
  const int tx = along_i ? IOFF + lo : IOFF + (low ? 0 : n - 4);
  const int ty = along_i ? JOFF + (low ? 1 : n - 4) : JOFF + lo;
  const uint32_t tbytes = (uint32_t)(nsrc * (along_i ? 3 : 4) * sp * sizeof(T));
  auto issue = [&](int kk, int slot) {                   // thread 0: both fields of plane kk
    uint64_t* bar = bars + slot;
    mbar_expect_tx(bar, tbytes);
    const CUtensorMap* m = along_i ? &a.mRow : &a.mCol;
    tma_load_3d(sm + slot * SLOT, m, tx, ty, zs0 + kk, bar);
    if (nsrc == 2) tma_load_3d(sm + slot * SLOT + FS, m, tx, ty, zs1 + kk, bar);
  };

  // spread piece (column sources): one row of one field per thread
  const bool spreader = !along_i && tid < nsrc * sp;
  const int spf = tid >= sp ? 1 : 0, spu = tid - spf * sp;
  const int sp_src = spf * FS + spu * 4, sp_dst = spf * FS + spu;
  // outputs: S/N receivers store rows directly; W/E receivers write sectors from `res`
  T* const dst0 = a.q + g.vol(run, face, ol0) + (long long)kb * g.plane;
  T* const dst1 = a.q + g.vol(run, face, ol1) + (long long)kb * g.plane;
  T* gout0 = dst0 + g.at(0, e == 0 ? -1 - l : n + l, valid ? t : 0);
  const long long gap = dst1 - dst0;                     // second output field
  const bool writer = cols && tid < ts && seg * ts + tid < n;
  T* sec0 = dst0 + g.at(0, writer ? seg * ts + tid : 0, e == 2 ? -SECT : n);
  // tap window inside a [layer][u] plane; row sources hold the layers in row order
  const int boff = (along_i && !low ? 2 - l : l) * sp + s0;

  auto spread = [&](int slot, int half) {                // [f][u][4] -> [f][layer][u]
    if (spreader) {
      T v[4];
      ldv(sm + slot * SLOT + sp_src, v);
      if (sizeof(T) == 8) ldv(sm + slot * SLOT + sp_src + 2, v + 2);
      T* d = tb + half * 2 * FS + sp_dst;
#pragma unroll
      for (int ll = 0; ll < 3; ++ll) d[ll * sp] = v[low ? 1 + ll : 2 - ll];
    }
  };
  auto put_sector = [&](T* d, const T* r) {
    T sect[SECT];
#pragma unroll
    for (int m = 0; m < SECT; ++m) sect[m] = T(0);
    if (e == 2) {
#pragma unroll
      for (int ll = 0; ll < 3; ++ll) sect[SECT - 1 - ll] = r[ll * ts];
    } else {
#pragma unroll
      for (int ll = 0; ll < 3; ++ll) sect[ll] = r[ll * ts];
    }
    st_sector(d, sect);
  };
  auto sectors = [&](int half) {                         // W/E: one whole sector per row
    if (writer) {
      const T* r = res + half * 6 * ts + tid;
      put_sector(sec0, r);
      if (nout == 2) put_sector(sec0 + gap, r + 3 * ts);
      sec0 += g.plane;
    }
  };

  if (tid == 0) {
    for (int s = 0; s < kEdgeRing; ++s) mbar_init(bars + s, 1);
    mbar_fence_init();
  }
  __syncthreads();
  // The previous kernel may still be finishing (programmatic launch): everything above
  // reads constant tables only; the buffer comes after the wait.
  grid_dependency_wait();
  // A thread whose wait gives up stops waiting and thread 0 stops issuing; the CTA leaves
  // the plane loop at the next barrier, and thread 0 waits for the planes it issued but did
  // not see land before the CTA exits.  fail_at = the plane whose wait thread 0 gave up on.
  if (tid == 0 && !a.wc.no_loads)
    for (int d = 0; d < kEdgeDepth && d < kc; ++d) issue(d, d);
  bool ok = mbar_wait(bars, 0, a.wc, kErrEdgeRing), failed = false;
  if (__syncthreads_or(!ok)) {
    // thread 0 issued the first kEdgeDepth planes and saw plane 0 land if its wait succeeded
    if (tid == 0 && !a.wc.no_loads) mbar_drain(bars, kEdgeRing, 0, ok ? 1 : 0, min(kEdgeDepth, kc), a.wc.polls);
    return;
  }
  spread(0, 0);
  int fail_at = kc;
  int kk = 0;
  int rs = 0;                                            // ring slot of plane kk
  int ws = kEdgeDepth;                                   // ring slot of plane kk + kEdgeDepth
  int ns = 1;                                            // ring slot of plane kk + 1 ...
  uint32_t np = 0;                                       // ... and the parity of its phase
  for (; kk < kc; ++kk) {
    if (tid == 0 && ok && !a.wc.no_loads && kk + kEdgeDepth < kc) issue(kk + kEdgeDepth, ws);
    ws = ws + 1 == kEdgeRing ? 0 : ws + 1;
    if (ns == 0) np ^= 1;
    if (ok && kk + 1 < kc && !mbar_wait(bars + ns, np, a.wc, kErrEdgeRing)) { ok = false; fail_at = kk + 1; }
    if (__syncthreads_or(!ok)) { failed = true; break; }
    if (kk > 0) sectors((kk - 1) & 1);
    if (kk + 1 < kc) spread(ns, (kk + 1) & 1);
    const T* b = (along_i ? sm + rs * SLOT : tb + (kk & 1) * 2 * FS) + boff;
    T r0, r1 = T(0);
    if (vec) {
      T a0 = T(0), a1 = T(0);
#pragma unroll
      for (int s = 0; s < 9; ++s) {
        a0 = fma(c0[s], b[s], a0);
        a1 = fma(c1[s], b[FS + s], a1);
      }
      r0 = a0 + a1;
    } else {
      T a0 = T(0), a1 = T(0);
#pragma unroll
      for (int s = 0; s < 9; s += 2) a0 = fma(c0[s], b[s], a0);
#pragma unroll
      for (int s = 1; s < 9; s += 2) a1 = fma(c0[s], b[s], a1);
      r0 = a0 + a1;
      if (nout == 2) {
        const T* b1 = b + FS;
        T a2 = T(0), a3 = T(0);
#pragma unroll
        for (int s = 0; s < 9; s += 2) a2 = fma(c0[s], b1[s], a2);
#pragma unroll
        for (int s = 1; s < 9; s += 2) a3 = fma(c0[s], b1[s], a3);
        r1 = a2 + a3;
      }
    }
    if (!cols) {
      if (valid) {
        *gout0 = r0;
        if (nout == 2) gout0[gap] = r1;
      }
      gout0 += g.plane;
    } else {
      T* rr = res + (kk & 1) * 6 * ts + l * ts + tl;
      rr[0] = r0;
      rr[3 * ts] = r1;
    }
    rs = ns;
    ns = ns + 1 == kEdgeRing ? 0 : ns + 1;
  }
  if (failed) {
    // at the break in iteration kk thread 0 had issued planes [0, kk + kEdgeDepth] and seen
    // [0, seen) land
    if (tid == 0 && !a.wc.no_loads) {
      const int issued = min(kk + kEdgeDepth + 1, kc);
      const int seen = min(fail_at, min(kk + 2, kc));
      mbar_drain(bars, kEdgeRing, 0, seen, issued, a.wc.polls);
    }
    return;
  }
  if (cols) {
    __syncthreads();
    sectors((kc - 1) & 1);
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
// grad_r, div) into the v_xi, v_eta, v_r, p slots of qout.  MODE 4 / 5: MODE 1 / 0 that
// also store the divergence of the stage input (compact, run 0) into divout -- the
// forward recomputation of the adjoint.
constexpr int kLead = 8;
// tile-ring depth: plane k is computed while planes k+1, k+2 are in flight
template <typename T> struct TileRing { static constexpr int value = 3; };

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
  T* divout;                // MODE 4/5: compact divergence [face][k][j][i]
  const T* force;           // FORCE: this step's forcing field [face][j][i] (v_r equation)
  const T* force_r;         // FORCE: its radial factor [nr]
  const int* runs;          // stored run of each launched run index, or nullptr
  WaitCtl wc;               // error word and bound of the ring waits
  Geom g;
  T dt, alpha, beta, inv_dxi;
  int kchunk;
  int tsel;                 // tiles launched: kTilesAll, kTilesInterior or kTilesRing
};

// Tile subsets of a face (stage_tile).  The interior tiles (1..tx-2) x (1..ty-2) read no
// ghost frame: their xi and eta halos lie inside the face.  The ring is the tiles along the
// four face edges.  A process that owns part of the sphere runs the interior tiles while
// the edge lines of the phase are still in transit, then the ring after the edge kernel.
enum TileSel { kTilesAll = 0, kTilesInterior = 1, kTilesRing = 2 };

// Tile (ix, iy) of launch index t among tx x ty tiles.  Interior and ring need tx, ty >= 3;
// the ring lists rows 0 and ty-1, then columns 0 and tx-1 of rows 1..ty-2.
__host__ __device__ inline void stage_tile(int tsel, int t, int tx, int ty, int* ix, int* iy) {
  if (tsel == kTilesInterior) {
    *ix = 1 + t % (tx - 2);
    *iy = 1 + t / (tx - 2);
  } else if (tsel == kTilesRing) {
    if (t < 2 * tx) {
      *ix = t % tx;
      *iy = t < tx ? 0 : ty - 1;
    } else {
      const int r = t - 2 * tx;
      *iy = 1 + r / 2;
      *ix = (r & 1) ? tx - 1 : 0;
    }
  } else {
    *ix = t % tx;
    *iy = t / tx;
  }
}
__host__ __device__ inline int stage_tile_count(int tsel, int tx, int ty) {
  if (tsel == kTilesInterior) return (tx - 2) * (ty - 2);
  if (tsel == kTilesRing) return 2 * tx + 2 * (ty - 2);
  return tx * ty;
}

template <typename T, int TX, int TY, bool HAS_RHO>
struct StageLayout {
  static constexpr int PB = (TX + 8) * (TY + 6), XB = (TX + 8) * TY, YB = TX * (TY + 6), OB = TX * TY;
  static constexpr int NO = HAS_RHO ? 6 : 4;                          // rho + qw boxes
  static constexpr size_t P_BYTES = align128(PB * sizeof(T));
  static constexpr size_t X_BYTES = align128(XB * sizeof(T));
  static constexpr size_t Y_BYTES = align128(YB * sizeof(T));
  static constexpr size_t O_BYTES = align128(OB * sizeof(T));
  static constexpr size_t LEAD = P_BYTES + O_BYTES;                    // p box + v_r
  static constexpr size_t TILE = X_BYTES + Y_BYTES + NO * O_BYTES;     // v_xi, v_eta, (rho), qw
  static constexpr int RING = TileRing<T>::value;
  static constexpr size_t BAR = kLead * LEAD + RING * TILE;
  static constexpr size_t TOTAL = BAR + (kLead + RING) * sizeof(uint64_t);
};

// Each thread owns V consecutive points of one row (V = 16 bytes / sizeof(T)), so the
// CTA has (TX/V) x TY threads and every shared-memory access is a 16-byte vector.
template <typename T, int TX, int TY, int MODE_, bool HAS_RHO, bool FORCE = false>
__global__ void __launch_bounds__((TX / Vec16<T>::V) * TY) stage_kernel(const __grid_constant__ StageArgs<T> a) {
  constexpr bool STORE_DIV = MODE_ >= 4;
  constexpr int MODE = MODE_ == 4 ? 1 : (MODE_ == 5 ? 0 : MODE_);
  constexpr int V = Vec16<T>::V;
  constexpr int kTile = TileRing<T>::value;
  constexpr int NT = TX / V;
  constexpr int NV = (V + 8) / V;            // vectors covering box columns c .. c+V+7
  constexpr int PW = TX + 8;
  constexpr int QOFF = HAS_RHO ? 1 : 0;      // first qw box inside a tile slot
  using L = StageLayout<T, TX, TY, HAS_RHO>;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* barL = reinterpret_cast<uint64_t*>(smem + L::BAR);
  uint64_t* barT = barL + kLead;
  const Geom& g = a.g;
  const int n = g.n, nr = g.nr;
  const int tiles_x = n / TX;
  int tix, tiy;
  stage_tile(a.tsel, blockIdx.x, tiles_x, n / TY, &tix, &tiy);
  const int i0 = tix * TX, j0 = tiy * TY;
  // the run map is written before the launches that use it and constant during them
  const int zr = blockIdx.z / g.nface;
  const int run = a.runs ? a.runs[zr] : zr, face = g.face0 + blockIdx.z % g.nface;
  const int kb = g.k0 + blockIdx.y * a.kchunk;
  if (kb >= g.k1) return;
  const int ke = min(g.k1, kb + a.kchunk);
  const int cx = threadIdx.x, ty = threadIdx.y, tid = ty * NT + cx;
  const int sP = g.slot[kP], sX = g.slot[kVxi], sY = g.slot[kVeta], sR = g.slot[kVr], sRho = g.slot[kRho];
  const int zbase = (run * 6 + face) * g.nf;   // plane index of (slot s, k) = (zbase + s) * nr + k
  auto clampk = [nr](int k) { return min(max(k - 3, 0), nr - 7); };
  const int m_lo = clampk(kb), m_hi = clampk(ke - 1) + 6;

  auto lead = [&](int slot) { return smem + slot * L::LEAD; };
  auto tile = [&](int slot) { return smem + kLead * L::LEAD + slot * L::TILE; };
  const int xP = IOFF + i0 - 4, yP = JOFF + j0 - 3;   // p / v_xi boxes start 4 columns left
  const int xO = IOFF + i0, yO = JOFF + j0;
  auto issue_lead = [&](int m, int slot) {
    uint64_t* b = &barL[slot];
    mbar_expect_tx(b, (L::PB + L::OB) * sizeof(T));
    tma_load_3d(lead(slot), &a.mP, xP, yP, (zbase + sP) * nr + m, b);
    tma_load_3d(lead(slot) + L::P_BYTES, &a.mO, xO, yO, (zbase + sR) * nr + m, b);
  };
  auto issue_tile = [&](int k, int slot) {
    uint64_t* b = &barT[slot];
    uint32_t bytes = (L::XB + L::YB) * sizeof(T);
    if (HAS_RHO && MODE != 3) bytes += L::OB * sizeof(T);
    if (MODE == 0) bytes += g.nf * L::OB * sizeof(T);
    mbar_expect_tx(b, bytes);
    unsigned char* t = tile(slot);
    tma_load_3d(t, &a.mX, xP, yO, (zbase + sX) * nr + k, b);
    tma_load_3d(t + L::X_BYTES, &a.mY, xO, yP, (zbase + sY) * nr + k, b);
    if (HAS_RHO && MODE != 3)
      tma_load_3d(t + L::X_BYTES + L::Y_BYTES, &a.mO, xO, yO, (zbase + sRho) * nr + k, b);
    if (MODE == 0)
      for (int s = 0; s < g.nf; ++s)
        tma_load_3d(t + L::X_BYTES + L::Y_BYTES + (QOFF + s) * L::O_BYTES, &a.mW, xO, yO, (zbase + s) * nr + k, b);
  };

  // per-point constants (constant tables: read before the dependency wait)
  const long long P2 = (long long)n * n;
  const int ib = i0 + V * cx, j = j0 + ty;
  const int p2 = j * n + ib;
  T m_D[V], m_XYD[V], m_C[V], m_XYC[V], m_DivX[V], m_DivY[V], m_TX[V], m_TY[V];
  ldv(a.met + mD * P2 + p2, m_D);
  ldv(a.met + mXYD * P2 + p2, m_XYD);
  ldv(a.met + mC * P2 + p2, m_C);
  ldv(a.met + mXYC * P2 + p2, m_XYC);
  ldv(a.met + mDivX * P2 + p2, m_DivX);
  ldv(a.met + mDivY * P2 + p2, m_DivY);
  ldv(a.met + mTX * P2 + p2, m_TX);
  ldv(a.met + mTY * P2 + p2, m_TY);
  const T c1 = Coef<T>::drp(1), c2 = Coef<T>::drp(2), c3 = Coef<T>::drp(3);
  if (tid == 0) {
    for (int q = 0; q < kLead + kTile; ++q) mbar_init(&barL[q], 1);
    mbar_fence_init();
  }
  __syncthreads();
  // The previous kernel may still be finishing (programmatic launch): everything above
  // reads constant tables only; the state and the source term come after the wait.
  grid_dependency_wait();
  // producer state (thread 0 only): lead planes [m_lo, m_issued) have loads issued
  int m_issued = m_lo, slot_issue = 0;
  const bool loads = !a.wc.no_loads;
  if (tid == 0 && loads) {
    tma_prefetch_desc(&a.mP);
    for (; m_issued <= min(m_lo + kLead - 1, m_hi); ++m_issued) {
      issue_lead(m_issued, slot_issue);
      if (++slot_issue == kLead) slot_issue = 0;
    }
    for (int k = kb; k < min(kb + kTile, ke); ++k) issue_tile(k, k - kb);
  }

  T f_xy[V];
  if (FORCE) ldv(a.force + (long long)face * P2 + p2, f_xy);
  const long long own = g.at(0, j, ib);
  T* outS[5];
  T* qwS[5];
#pragma unroll
  for (int f = 0; f < 5; ++f) {
    const int sl = g.slot[f] < 0 ? 0 : g.slot[f];
    outS[f] = a.qout + g.vol(run, face, sl) + own;
    qwS[f] = a.qw + g.vol(run, face, sl) + own;
  }
  const int pc = (ty + 3) * PW + V * cx;       // box row of the own points; own point q at column V*cx+4+q
  const int xc = ty * PW + V * cx;
  const int yc = (ty + 3) * TX + V * cx;
  const int oc = ty * TX + V * cx;

  // radial coefficients of the current plane; the next plane's are loaded one iteration
  // ahead so their latency hides behind the compute
  struct Rad { T facr, invr, rho0, inv_rho0, c2rho0, rho0g0, sig, drho0, g0rho0, frc; };
  auto load_rad = [&](int k) {
    Rad r;
    r.frc = FORCE ? __ldg(a.force_r + k) : T(0);
    r.facr = __ldg(a.rad + rFacR * nr + k);
    r.invr = __ldg(a.rad + rInvR * nr + k);
    r.rho0 = __ldg(a.rad + rRho0 * nr + k);
    r.inv_rho0 = __ldg(a.rad + rInvRho0 * nr + k);
    r.c2rho0 = __ldg(a.rad + rC2Rho0 * nr + k);
    r.rho0g0 = __ldg(a.rad + rRho0G0 * nr + k);
    r.sig = __ldg(a.rad + rSigma * nr + k);
    r.drho0 = HAS_RHO ? __ldg(a.rad + rDRho0 * nr + k) : T(0);
    r.g0rho0 = HAS_RHO ? __ldg(a.rad + rG0Rho0 * nr + k) : T(0);
    return r;
  };
  Rad rc = load_rad(kb);
  T pw[7][V], vw[7][V];
#pragma unroll
  for (int s = 0; s < 7; ++s)
#pragma unroll
    for (int q = 0; q < V; ++q) { pw[s][q] = T(0); vw[s][q] = T(0); }
  int mq = m_lo, slot_q = 0, slot_k = (kb - m_lo) % kLead, slot_t = 0;
  uint32_t phase_q = 0, phase_t = 0;
  // A thread whose wait gives up stops waiting; the CTA leaves at the barrier that closes
  // the iteration, and thread 0 waits for what it issued but did not see land before the
  // CTA exits.  lead_fail = the lead plane whose wait thread 0 gave up on; tile_fail = its
  // tile wait gave up.
  bool ok = true, failed = false, tile_fail = false;
  int lead_fail = 0x7fffffff;
  int k = kb;
  for (; k < ke; ++k) {
    const int ks = clampk(k);
    for (; mq <= ks + 6; ++mq) {
      if (ok && !mbar_wait(&barL[slot_q], phase_q, a.wc, kErrStageLead)) { ok = false; lead_fail = mq; }
      const T* bp = reinterpret_cast<const T*>(lead(slot_q));
#pragma unroll
      for (int s = 0; s < 6; ++s)
#pragma unroll
        for (int q = 0; q < V; ++q) { pw[s][q] = pw[s + 1][q]; vw[s][q] = vw[s + 1][q]; }
      ldv(bp + pc + 4, pw[6]);
      ldv(reinterpret_cast<const T*>(lead(slot_q) + L::P_BYTES) + oc, vw[6]);
      if (++slot_q == kLead) { slot_q = 0; phase_q ^= 1; }
    }
    if (ok && !mbar_wait(&barT[slot_t], phase_t, a.wc, kErrStageTile)) { ok = false; tile_fail = true; }
    const Rad rn = load_rad(min(k + 1, nr - 1));
    const T* sp = reinterpret_cast<const T*>(lead(slot_k));
    const unsigned char* tb = tile(slot_t);
    const T* sx = reinterpret_cast<const T*>(tb);
    const T* sy = reinterpret_cast<const T*>(tb + L::X_BYTES);
    // xi windows of p and v_xi; eta columns of p and v_eta
    T wp[NV * V], wx[NV * V];
#pragma unroll
    for (int m = 0; m < NV; ++m) { ldv(sp + pc + m * V, wp + m * V); ldv(sx + xc + m * V, wx + m * V); }
    T pu[3][V], pd[3][V], yu[3][V], yd[3][V], vyo[V];
#pragma unroll
    for (int d = 1; d <= 3; ++d) {
      ldv(sp + pc + 4 + d * PW, pu[d - 1]);
      ldv(sp + pc + 4 - d * PW, pd[d - 1]);
      ldv(sy + yc + d * TX, yu[d - 1]);
      ldv(sy + yc - d * TX, yd[d - 1]);
    }
    ldv(sy + yc, vyo);
    T rho[V], qwv[5][V];
    if (HAS_RHO && MODE != 3) ldv(reinterpret_cast<const T*>(tb + L::X_BYTES + L::Y_BYTES) + oc, rho);
    if (MODE == 0)
#pragma unroll
      for (int f = 0; f < 5; ++f)
        if (f != kRho || HAS_RHO) {
          const int sl = HAS_RHO ? f : f - 1;
          ldv(reinterpret_cast<const T*>(tb + L::X_BYTES + L::Y_BYTES + (QOFF + sl) * L::O_BYTES) + oc, qwv[f]);
        }
    const T facr = rc.facr;
    const T invr = rc.invr;
    const bool interior = k >= 3 && k <= nr - 4;
    const int offk = k - ks;
    const int brow = k < 3 ? k : nr - 1 - k;
    T r_p[V], r_vx[V], r_ve[V], r_vr[V], r_rho[V], vr[V], pv[V], vxv[V];
    T o0[V], o1[V], o2[V], o3[V], dvv[V];
#pragma unroll
    for (int q = 0; q < V; ++q) {
      const T dpx = a.inv_dxi * (c1 * (wp[5 + q] - wp[3 + q]) + c2 * (wp[6 + q] - wp[2 + q]) + c3 * (wp[7 + q] - wp[1 + q]));
      const T dpy = a.inv_dxi * (c1 * (pu[0][q] - pd[0][q]) + c2 * (pu[1][q] - pd[1][q]) + c3 * (pu[2][q] - pd[2][q]));
      const T dvx = a.inv_dxi * (c1 * (wx[5 + q] - wx[3 + q]) + c2 * (wx[6 + q] - wx[2 + q]) + c3 * (wx[7 + q] - wx[1 + q]));
      const T dvy = a.inv_dxi * (c1 * (yu[0][q] - yd[0][q]) + c2 * (yu[1][q] - yd[1][q]) + c3 * (yu[2][q] - yd[2][q]));
      T dpr, dvr, v_r;
      if (interior) {
        dpr = facr * (c1 * (pw[4][q] - pw[2][q]) + c2 * (pw[5][q] - pw[1][q]) + c3 * (pw[6][q] - pw[0][q]));
        dvr = facr * (c1 * (vw[4][q] - vw[2][q]) + c2 * (vw[5][q] - vw[1][q]) + c3 * (vw[6][q] - vw[0][q]));
        v_r = vw[3][q];
      } else {
        const bool lo = k < 3;
        T a_ = T(0), b_ = T(0);
#pragma unroll
        for (int s = 0; s < 7; ++s) {
          const T b = Coef<T>::bdy(brow, lo ? s : 6 - s);
          a_ = fma(b, pw[s][q], a_);
          b_ = fma(b, vw[s][q], b_);
        }
        dpr = lo ? facr * a_ : -facr * a_;
        dvr = lo ? facr * b_ : -facr * b_;
        v_r = vw[0][q];
#pragma unroll
        for (int s = 1; s < 7; ++s) v_r = (offk == s) ? vw[s][q] : v_r;
      }
      const T p = wp[4 + q], vxi = wx[4 + q], veta = vyo[q];
      const T gxi = invr * (m_D[q] * dpx + m_XYD[q] * dpy);
      const T geta = invr * (m_C[q] * dpy + m_XYC[q] * dpx);
      const T div = invr * (m_DivX[q] * dvx + m_DivY[q] * dvy - m_TX[q] * vxi - m_TY[q] * veta) + dvr + T(2) * v_r * invr;
      vr[q] = v_r; pv[q] = p; vxv[q] = vxi;
      if (STORE_DIV) dvv[q] = div;
      if (MODE == 3) {
        o0[q] = gxi; o1[q] = geta; o2[q] = dpr; o3[q] = div;
      } else {
        const T rho0 = rc.rho0, inv_rho0 = rc.inv_rho0;
        T c2rho0 = rc.c2rho0;
        if (a.c2) c2rho0 = a.c2[((long long)face * nr + k) * P2 + p2 + q] * rho0;
        r_vx[q] = -gxi * inv_rho0;
        r_ve[q] = -geta * inv_rho0;
        r_vr[q] = -dpr * inv_rho0;
        r_p[q] = -c2rho0 * div + rc.rho0g0 * v_r;
        if (HAS_RHO) {
          r_rho[q] = -rho0 * div - v_r * rc.drho0;
          r_vr[q] -= rho[q] * rc.g0rho0;
        }
        if (FORCE) r_vr[q] += f_xy[q] * rc.frc;         // + S(theta, phi, t) e_r
      }
    }
    const long long kp = (long long)k * g.plane;
    if (STORE_DIV) stv(a.divout + ((long long)face * nr + k) * P2 + p2, dvv);
    if (MODE == 3) {
      stv(outS[kVxi] + kp, o0);
      stv(outS[kVeta] + kp, o1);
      stv(outS[kVr] + kp, o2);
      stv(outS[kP] + kp, o3);
    } else if (MODE == 2) {
      if (HAS_RHO) stv(outS[kRho] + kp, r_rho);
      stv(outS[kVxi] + kp, r_vx);
      stv(outS[kVeta] + kp, r_ve);
      stv(outS[kVr] + kp, r_vr);
      stv(outS[kP] + kp, r_p);
    } else {
      // BC_RHS (bc_acoustic_wave.f90:14-34) then SPONGE (sponge.f90:40-50)
      const bool bc = (k == 0 || k == nr - 1);
      const T sig = rc.sig;
      const T dt = a.dt, alpha = a.alpha, beta = a.beta;
      // qw = alpha qw + dt rhs ; q = q + beta qw   (timestep.f90:68-69)
      auto update = [&](int f, const T* qv, const T* rv, bool damped) {
        T w[V], o[V];
#pragma unroll
        for (int q = 0; q < V; ++q) {
          T r = bc ? T(0) : rv[q];
          if (damped) r -= sig * qv[q];
          w[q] = (MODE == 1) ? dt * r : fma(alpha, qwv[f][q], dt * r);
          o[q] = fma(beta, w[q], qv[q]);
        }
        stv(qwS[f] + kp, w);
        stv(outS[f] + kp, o);
      };
      if (HAS_RHO) update(kRho, rho, r_rho, true);
      update(kVxi, vxv, r_vx, false);
      update(kVeta, vyo, r_ve, false);
      update(kVr, vr, r_vr, true);
      update(kP, pv, r_p, true);
    }
    // every thread is done with lead plane k and tile plane k: refill their slots
    if (__syncthreads_or(!ok)) { failed = true; break; }
    if (tid == 0 && loads) {
      if (k + kTile < ke) issue_tile(k + kTile, slot_t);
      for (; m_issued <= min(k + kLead, m_hi); ++m_issued) {
        issue_lead(m_issued, slot_issue);
        if (++slot_issue == kLead) slot_issue = 0;
      }
    }
    if (++slot_t == kTile) { slot_t = 0; phase_t ^= 1; }
    if (++slot_k == kLead) slot_k = 0;
    rc = rn;
  }
  if (failed && tid == 0 && loads) {
    // at the break in iteration k: tile planes [kb, min(k + kTile, ke)) were issued and
    // thread 0 saw [kb, k + 1) land unless one of its waits in this iteration gave up
    const bool own_fail = lead_fail != 0x7fffffff || tile_fail;
    mbar_drain(barL, kLead, m_lo, min(lead_fail, mq), m_issued, a.wc.polls);
    mbar_drain(barT, kTile, kb, own_fail ? k : k + 1, min(k + kTile, ke), a.wc.polls);
  }
}

// ---------------------------------------------------------------------------------
// Filter kernel: FILTER_EXP for one field (filter.f90:9-48): xi filter of q (with the
// q halos), eta filter of that (rows outside the face take the UNFILTERED q halo,
// filter.f90:43), 11-point radial filter of the result; the 5 end planes at each radial
// end become 0 (filter.f90:726-775).  A CTA owns a TX x TY column tile of one face and
// one field and streams every plane through a kFilt-deep TMA ring, keeping the last 11
// eta-filtered values of its column in registers.  When the whole-column CTAs leave the
// last wave of the GPU partly empty, the remaining columns are cut into radial chunks
// (each re-reading the 5 planes on either side) that fill that wave.
constexpr int kFiltRing = 4;

template <typename T>
struct FilterArgs {
  CUtensorMap mP;           // input buffer, box (TX+8) x (TY+6)
  T* qout;
  const int* runs;          // stored run of each launched run index, or nullptr
  WaitCtl wc;               // error word and bound of the ring waits
  Geom g;
  int whole;                // CTAs 0 .. whole-1 filter one (tile, field, face, run) unit each
  int chunks;               // later CTAs filter one of `chunks` radial chunks of a unit
};

template <typename T, int TX, int TY>
struct FilterLayout {
  static constexpr int PB = (TX + 8) * (TY + 6), SB = (TY + 6) * TX;
  static constexpr size_t P_BYTES = align128(PB * sizeof(T));
  static constexpr size_t S_BYTES = align128(SB * sizeof(T));
  static constexpr size_t BAR = kFiltRing * P_BYTES + 2 * S_BYTES;
  static constexpr size_t TOTAL = BAR + kFiltRing * sizeof(uint64_t);
};

// Each thread owns V consecutive points (V = 16 bytes / sizeof(T)) in each of R consecutive
// rows; the CTA has (TX/V) x (TY/R) threads.  Per plane: every thread xi-filters its own R
// rows of the box (rows outside the face keep the unfiltered halo), keeps them in registers
// and stores them to shared memory with 16-byte stores, and the first thread rows also
// filter the 6 halo rows of the box.  After one barrier each thread reads the 3 xi-filtered
// rows above and the 3 below its own, eta-filters its R x V points and pushes them into an
// 11-deep register queue; the k loop is unrolled by 11 so the queue indices are constants.
// With R = 2 a thread reads 6 rows from shared memory for 2 output rows instead of 7 for 1.
// The float kernel's bound of four CTAs per SM lets the compiler use 91 registers: at 6 x
// 128^3 it ran in 100 us against 106 us at 88 registers (a bound of five) and 115 us at 83
// (no bound).  The filter weights are compile-time values (scheme.h).
template <typename T, int TX, int TY, int R>
__global__ void __launch_bounds__((TX / Vec16<T>::V) * (TY / R), sizeof(T) == 4 ? 4 : 1) filter_kernel(const __grid_constant__ FilterArgs<T> a) {
  constexpr int V = Vec16<T>::V;
  constexpr int NT = TX / V;                 // threads per row
  constexpr int NY = TY / R;                 // thread rows
  constexpr int NV = (V + 8) / V;            // vectors covering columns c-4 .. c+V+3
  constexpr int NP = V / 2;                  // float pairs per row (float only)
  static_assert(TY % R == 0, "the rows per thread divide the tile height");
  using L = FilterLayout<T, TX, TY>;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L::BAR);
  const Geom& g = a.g;
  const int n = g.n, nr = g.nr;
  const int tiles_x = n / TX, tiles = tiles_x * (n / TY);
  // unit = (tile, stored field, run and owned face); whole units first, then the radial
  // chunks of the remaining units (output planes [ko0, ko1), input planes [ks, ke))
  int unit = blockIdx.x, ko0 = g.k0, ko1 = g.k1;
  if (unit >= a.whole) {
    const int t = unit - a.whole, c = t % a.chunks, nk = g.k1 - g.k0;
    unit = a.whole + t / a.chunks;
    ko0 = g.k0 + c * nk / a.chunks;
    ko1 = g.k0 + (c + 1) * nk / a.chunks;
  }
  const int ks = max(0, ko0 - 5), ke = min(nr, ko1 + 5);
  const int tile = unit % tiles, rest = unit / tiles;
  const int i0 = (tile % tiles_x) * TX, j0 = (tile / tiles_x) * TY;
  const int s = rest % g.nf;                 // stored field
  const int rz = rest / g.nf;
  const int run = a.runs ? a.runs[rz / g.nface] : rz / g.nface, face = g.face0 + rz % g.nface;
  const int cx = threadIdx.x, ty = threadIdx.y, tid = ty * NT + cx;
  const int rb = R * ty;                     // first own row of the tile
  constexpr int PW = TX + 8;
  const int z0 = ((run * 6 + face) * g.nf + s) * nr;
  const int xP = IOFF + i0 - 4, yP = JOFF + j0 - 3;
  auto issue = [&](int k, int slot) {
    uint64_t* b = &bars[slot];
    mbar_expect_tx(b, L::PB * sizeof(T));
    tma_load_3d(smem + slot * L::P_BYTES, &a.mP, xP, yP, z0 + k, b);
  };
  if (tid == 0) {
    for (int q = 0; q < kFiltRing; ++q) mbar_init(&bars[q], 1);
    mbar_fence_init();
  }
  __syncthreads();
  // The previous kernel may still be finishing (programmatic launch): the input is read
  // only after the wait.
  grid_dependency_wait();
  const bool loads = !a.wc.no_loads;
  if (tid == 0 && loads)
    for (int k = ks; k < min(ks + kFiltRing, ke); ++k) issue(k, k - ks);
  T* out = a.qout + g.vol(run, face, s) + g.at(0, j0 + rb, i0 + V * cx);
  constexpr T f0 = T(kFilt[0]), f1 = T(kFilt[1]), f2 = T(kFilt[2]), f3 = T(kFilt[3]);
  constexpr T rw[6] = {T(kFiltR[0]), T(kFiltR[1]), T(kFiltR[2]), T(kFiltR[3]), T(kFiltR[4]), T(kFiltR[5])};
  // xi filter of box row r (tile row r - 3) at columns V*cx .. V*cx+V-1 of the tile
  auto xi_row = [&](const T* bx, int r, T* v) {
    const int jr = j0 - 3 + r;
    T w[NV * V];
#pragma unroll
    for (int m = 0; m < NV; ++m) ldv(bx + r * PW + V * cx + m * V, w + m * V);
    // w[q'] holds box column V*cx + q'; the own point q sits at box column V*cx + 4 + q
    constexpr int o = 4;
    if (jr < 0 || jr >= n) {
#pragma unroll
      for (int q = 0; q < V; ++q) v[q] = w[o + q];
    } else {
#pragma unroll
      for (int q = 0; q < V; ++q)
        v[q] = f0 * w[o + q] + f1 * (w[o + q - 1] + w[o + q + 1]) + f2 * (w[o + q - 2] + w[o + q + 2]) +
               f3 * (w[o + q - 3] + w[o + q + 3]);
    }
  };
  // radial queue of eta-filtered planes; in float the V values of a thread's row are held
  // as packed pairs and the eta and radial filters run on pairs
  constexpr bool PAIRS = sizeof(T) == 4;
  T tq[11][R][V];
  unsigned long long tq2[11][R][NP > 0 ? NP : 1];
#pragma unroll
  for (int m = 0; m < 11; ++m)
#pragma unroll
    for (int r = 0; r < R; ++r) {
#pragma unroll
      for (int q = 0; q < V; ++q) tq[m][r][q] = T(0);
#pragma unroll
      for (int h = 0; h < (NP > 0 ? NP : 1); ++h) tq2[m][r][h] = 0ull;
    }
  T zero[V];
#pragma unroll
  for (int q = 0; q < V; ++q) zero[q] = T(0);
  // A thread whose wait gives up reports it at the CTA barrier after the xi pass; the CTA
  // leaves the plane loop there, and thread 0 waits for the planes it issued but did not
  // see land (fail_at = 2 * plane + whether thread 0's own wait on that plane succeeded).
  bool ok = true;
  int fail_at = 0;
  int slot = 0;
  uint32_t phase = 0;
  for (int kb = ks; kb < ke && ok; kb += 11) {
#pragma unroll
    for (int u = 0; u < 11; ++u) {
      const int k = kb + u;
      if (k >= ke) break;
      const bool got = mbar_wait(&bars[slot], phase, a.wc, kErrFilterRing);
      const T* bx = reinterpret_cast<const T*>(smem + slot * L::P_BYTES);
      T* t1 = reinterpret_cast<T*>(smem + kFiltRing * L::P_BYTES + (k & 1) * L::S_BYTES);
      // c[m] holds xi-filtered box row rb + m (tile row rb - 3 + m)
      T c[R + 6][V];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        xi_row(bx, rb + 3 + r, c[3 + r]);
        stv(t1 + (rb + 3 + r) * TX + V * cx, c[3 + r]);
      }
      // the halo rows of the box: 0..2 and TY+3..TY+5
      for (int h = ty; h < 6; h += NY) {
        const int r = h < 3 ? h : TY + h;
        T v[V];
        xi_row(bx, r, v);
        stv(t1 + r * TX + V * cx, v);
      }
      if (__syncthreads_or(!got)) { ok = false; fail_at = 2 * k + (got ? 1 : 0); break; }
      if (tid == 0 && loads && k + kFiltRing < ke) issue(k + kFiltRing, slot);
      if (++slot == kFiltRing) { slot = 0; phase ^= 1; }
#pragma unroll
      for (int m = 0; m < 3; ++m) {
        ldv(t1 + (rb + m) * TX + V * cx, c[m]);
        ldv(t1 + (rb + R + 3 + m) * TX + V * cx, c[R + 3 + m]);
      }
      // eta filter of own row r: rows r .. r+6 of c
#pragma unroll
      for (int r = 0; r < R; ++r) {
        if constexpr (PAIRS) {
#pragma unroll
          for (int h = 0; h < NP; ++h) {
            auto pr = [&](int m) { return pk2(c[r + m][2 * h], c[r + m][2 * h + 1]); };
            unsigned long long t = mul2(pk2(f0, f0), pr(3));
            t = fma2(pk2(f1, f1), add2(pr(2), pr(4)), t);
            t = fma2(pk2(f2, f2), add2(pr(1), pr(5)), t);
            tq2[u][r][h] = fma2(pk2(f3, f3), add2(pr(0), pr(6)), t);
          }
        } else {
#pragma unroll
          for (int q = 0; q < V; ++q)
            tq[u][r][q] = f0 * c[r + 3][q] + f1 * (c[r + 2][q] + c[r + 4][q]) + f2 * (c[r + 1][q] + c[r + 5][q]) +
                          f3 * (c[r][q] + c[r + 6][q]);
        }
      }
      if (k - ks >= 10) {
        // planes k-10 .. k sit at queue rows (u+1 .. u+11) % 11; the centre is k-5
#pragma unroll
        for (int r = 0; r < R; ++r) {
          T v[V];
          if constexpr (PAIRS) {
#pragma unroll
            for (int h = 0; h < NP; ++h) {
              unsigned long long acc = mul2(pk2(rw[0], rw[0]), tq2[(u + 6) % 11][r][h]);
#pragma unroll
              for (int m = 1; m <= 5; ++m) {
                acc = fma2(pk2(rw[m], rw[m]), add2(tq2[(u + 6 - m) % 11][r][h], tq2[(u + 6 + m) % 11][r][h]), acc);
              }
              float x, y;
              upk2(acc, x, y);
              v[2 * h] = x;
              v[2 * h + 1] = y;
            }
          } else {
#pragma unroll
            for (int q = 0; q < V; ++q) {
              T acc = rw[0] * tq[(u + 6) % 11][r][q];
#pragma unroll
              for (int m = 1; m <= 5; ++m)
                acc += rw[m] * (tq[(u + 6 - m) % 11][r][q] + tq[(u + 6 + m) % 11][r][q]);
              v[q] = acc;
            }
          }
          stv(out + (long long)(k - 5) * g.plane + r * g.pitch, v);
        }
      }
    }
  }
  // the five end planes at each radial end are zero (filter.f90:726-775)
  for (int m = 0; m < 10; ++m) {
    const int k = m < 5 ? m : nr - 10 + m;
    if (k >= ko0 && k < ko1)
#pragma unroll
      for (int r = 0; r < R; ++r) stv(out + (long long)k * g.plane + r * g.pitch, zero);
  }
  if (!ok && tid == 0 && loads) {
    // at the break on plane k, planes [ks, min(k + kFiltRing, ke)) were issued
    const int k = fail_at >> 1;
    mbar_drain(bars, kFiltRing, ks, k + (fail_at & 1), min(k + kFiltRing, ke), a.wc.polls);
  }
}

// Edge lines exchanged between processes that own different zones: for item q the
// (zone, edge) pair items[2q], items[2q+1]; the three lines next to that edge that the
// neighbouring zone interpolates from (rows 1..3 / n-2..n-4, columns likewise), for the
// slots listed in `slots`, over the owned planes k0 .. k1-1.  Packed layout
// [item][slot][k - k0][layer][t], t along the edge.
template <typename T>
__device__ __forceinline__ long long line_offset(const Geom& g, int face, int e, int s, int k, int l, int t) {
  const int n = g.n;
  int ii, jj;
  if (e == 0) { ii = t; jj = l + 1; }
  else if (e == 1) { ii = t; jj = n - 2 - l; }
  else if (e == 2) { ii = l + 1; jj = t; }
  else { ii = n - 2 - l; jj = t; }
  return g.vol(0, face, s) + g.at(k, jj, ii);
}

template <typename T>
__global__ void line_pack_kernel(const T* __restrict__ q, T* __restrict__ out, const int* __restrict__ items,
                                 int nitems, const int* __restrict__ slots, int nslots, Geom g, int unpack) {
  const int nk = g.k1 - g.k0;                                // owned planes
  const long long per = (long long)3 * g.n * nk;             // one slot of one item
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= per * nslots * nitems) return;
  const int t = idx % g.n;
  long long r = idx / g.n;
  const int l = r % 3; r /= 3;
  const int k = g.k0 + (int)(r % nk); r /= nk;
  const int si = r % nslots;
  const int it = (int)(r / nslots);
  const long long o = line_offset<T>(g, items[2 * it], items[2 * it + 1], slots[si], k, l, t);
  if (unpack) const_cast<T*>(q)[o] = out[idx];
  else out[idx] = q[o];
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

// FP32 contexts: the compact volume is uploaded as float (rounded on the host).
__global__ void unpack_f32_kernel(const float* __restrict__ src, float* __restrict__ dst, Geom g) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long V = (long long)g.n * g.n * g.nr;
  if (idx >= V) return;
  const int i = idx % g.n, j = (idx / g.n) % g.n, k = idx / ((long long)g.n * g.n);
  dst[g.at(k, j, i)] = src[idx];
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
// Sum of squares of one stored field, for the per-step norm (auxiliary.f90:100-125): one
// CTA per (owned face, plane) adds its plane in FP64 (a warp per row, 16-byte loads) and
// writes one partial; sumsq_final_kernel adds the partials in a fixed order.
template <typename T>
__global__ void sumsq_plane_kernel(const T* __restrict__ q, Geom g, int run, int slot, double* part) {
  constexpr int V = Vec16<T>::V;
  const int nk = g.k1 - g.k0;
  const int face = g.face0 + blockIdx.x / nk, k = g.k0 + blockIdx.x % nk;
  const int n = g.n, per_row = n / V;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const T* base = q + g.vol(run, face, slot) + g.at(k, 0, 0);
  double acc = 0.0;
  for (int j = warp; j < n; j += nwarp) {
    const T* row = base + (long long)j * g.pitch;
    for (int c = lane; c < per_row; c += 32) {
      T v[V];
      ldv(row + c * V, v);
#pragma unroll
      for (int m = 0; m < V; ++m) acc = fma((double)v[m], (double)v[m], acc);
    }
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  __shared__ double red[32];
  if (lane == 0) red[warp] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < nwarp; ++w) t += red[w];
    part[blockIdx.x] = t;
  }
}

__global__ void sumsq_final_kernel(const double* __restrict__ part, int nblocks, double* out) {
  __shared__ double red[256];
  double acc = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) acc += part[b];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if ((int)threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = red[0];
}

// ---------------------------------------------------------------------------------
// NaN/Inf watchdog: scans the stored volumes of the owned zones of every run of one buffer
// (interior, ghost frame and padding -- the frame holds values interpolated from interiors,
// the padding zeros) with 16-byte loads.  The first launch that sees a non-finite value
// records its step number in *step_word; later ones leave it.  grid.y = volume
// ((run * nface + owned face) * nf + slot); grid.x strides over the volume.
template <typename T>
__global__ void __launch_bounds__(256) nonfinite_kernel(const T* __restrict__ q, Geom g, int step, int* step_word) {
  constexpr int V = Vec16<T>::V;
  const int y = blockIdx.y;
  const int s = y % g.nf, fz = (y / g.nf) % g.nface, run = y / (g.nf * g.nface);
  const T* base = q + g.vol(run, g.face0 + fz, s);
  const long long nv = g.vs / V;
  bool bad = false;
  for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += (long long)gridDim.x * blockDim.x) {
    T x[V];
    ldv(base + v * V, x);
#pragma unroll
    for (int m = 0; m < V; ++m) bad |= !isfinite(x[m]);
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicCAS(step_word, 0, step);
}

// ---------------------------------------------------------------------------------
// FP64 reductions for the diagnostics.  Stage 1: one CTA per (face, k) plane writes
// 5 partials; stage 2: one CTA sums them in a fixed order (deterministic).
//   part[0] = sum f_sel^2, [1] = energy, [2] = mass, [3] = max |p|, [4] = non-finite count
template <typename T>
__global__ void reduce_plane_kernel(const T* q, Geom g, int run, int sel_slot, const double* rad64,
                                    const double* vol2, const double* drw, const double* c2_3d,
                                    double* part) {
  const int nk = g.k1 - g.k0;
  const int face = g.face0 + blockIdx.x / nk, k = g.k0 + blockIdx.x % nk;
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


}  // namespace solar
