// adjoint_host.cuh -- host side of the discrete adjoint: receivers, checkpointed reverse
// sweep and the C-ABI entry points declared in include/solar_gpu.h.  Included once, by
// solar_gpu.cu: the adjoint kernels read the scheme constants that live in that
// translation unit's constant memory.
#pragma once

#include "adjoint.cuh"

namespace solar {

static long long state_bytes(const solar_ctx* c) { return 6LL * c->g.nf * c->g.vs * (long long)c->esize; }

static int adj_alloc(solar_ctx* c) {
  AdjBuffers& b = c->adj;
  if (c->g.nface != 6) return fail(SOLAR_ERR_ARG, "the adjoint entry points need a context owning all six zones");
  if (b.L) return SOLAR_OK;
  if (c->g.nruns != 1) return fail(SOLAR_ERR_ARG, "the adjoint entry points need nruns == 1");
  const size_t S = (size_t)state_bytes(c);
  void** bufs[4] = {&b.L, &b.LW, &b.T1, &b.T2};
  for (void** p : bufs) {
    if (cudaMalloc(p, S) != cudaSuccess) { cudaGetLastError(); return fail(SOLAR_ERR_NOMEM, "adjoint buffers: out of device memory"); }
    CK(cudaMemsetAsync(*p, 0, S, c->stream));
  }
  CK(cudaMalloc((void**)&b.grad, (size_t)6 * vol_compact(c) * sizeof(double)));
  CK(cudaMalloc(&b.rb, (size_t)6 * 4 * 2 * c->g.n * c->g.n * c->esize));
  CK(cudaMalloc((void**)&b.tspan, c->ht.tspan.size() * sizeof(int)));
  CK(cudaMemcpy(b.tspan, c->ht.tspan.data(), c->ht.tspan.size() * sizeof(int), cudaMemcpyHostToDevice));
  // Edge weights transposed to the gather's order: wt[kind][row][j][u] is the coefficient
  // with which ghost point t = lo(u) + j of row (face-edge, layer) used source position u
  // (kind 0: scalar weight, 1 and 2: the vector pair); zero past the ghost range of u.
  const int n = c->g.n;
  int span = 1;
  for (size_t q = 0; q < c->ht.tspan.size(); q += 2) span = std::max(span, c->ht.tspan[q + 1] - c->ht.tspan[q] + 1);
  std::vector<double> wt((size_t)3 * 72 * span * n, 0.0);
  for (int row = 0; row < 72; ++row)
    for (int u = 0; u < n; ++u) {
      const int lo = c->ht.tspan[((size_t)row * n + u) * 2], hi = c->ht.tspan[((size_t)row * n + u) * 2 + 1];
      for (int t = lo; t <= hi; ++t) {
        const int s = u - c->ht.s0t[(size_t)row * n + t];
        if (s < 0 || s > 8) continue;
        const size_t tap = (size_t)row * 9 + s, o = ((size_t)row * span + (t - lo)) * n + u;
        wt[o] = c->ht.ew[tap * n + t];
        wt[(size_t)72 * span * n + o] = c->ht.eg[(tap * 2 + 0) * n + t];
        wt[(size_t)2 * 72 * span * n + o] = c->ht.eg[(tap * 2 + 1) * n + t];
      }
    }
  int rc = c->fp32 ? upload<float>(&b.wt, wt) : upload<double>(&b.wt, wt);
  if (rc) return rc;
  b.wt_span = span;
  return SOLAR_OK;
}

// Grow-only device arrays of the adjoint (checkpoints, stage divergences, traces).
static int adj_reserve(void** p, size_t* have, size_t want) {
  if (*have >= want) return SOLAR_OK;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *have = 0;
  if (cudaMalloc(p, want) != cudaSuccess) {
    cudaGetLastError();
    return fail(SOLAR_ERR_NOMEM, "adjoint: cannot allocate %.2f GB of device memory", want / 1e9);
  }
  *have = want;
  return SOLAR_OK;
}

template <typename T>
static AdjStageArgs<T> adj_args(solar_ctx* c, double dt) {
  AdjStageArgs<T> a;
  a.lout = nullptr;
  a.lwout = nullptr;
  a.rb = nullptr;
  a.div = nullptr;
  a.c2 = (const T*)c->dt.c2;
  a.grad = nullptr;
  a.rad = (const T*)c->dt.rad;
  a.met = (const T*)c->dt.met;
  a.radT = (const T*)c->dt.radT;
  a.g = c->g;
  a.alpha = T(0);
  a.beta = T(1);
  a.dt = (T)dt;
  a.inv_dxi = (T)(1.0 / c->ht.dxi);
  a.keep = 0;
  a.kchunk = 0;
  a.wc = wait_ctl(c, kInjAdjStage);
  return a;
}

static unsigned blocks_for(long long n, int threads) { return (unsigned)((n + threads - 1) / threads); }

// L^T applied to buffer L (plus the pointwise and RK parts selected by `a`): the fused
// transposed stage writes lambda_q and lambda_w to the partner buffers T1, T2 (inputs'
// halos are read by neighbouring CTAs), the one-sided radial rows are added, the ghost
// adjoints are scattered back, and the buffer pairs swap roles.
template <typename T, int TX, int TY>
static int launch_adj_stage(solar_ctx* c, AdjStageArgs<T>& a) {
  using L = AdjLayout<T, TX, TY>;
  AdjBuffers& b = c->adj;
  if (!make_map(c, b.L, TX + 8, TY + 6, &a.mBq) || !make_map(c, b.LW, TX + 8, TY + 6, &a.mBw) ||
      !make_map(c, b.L, TX, TY, &a.mTq) || !make_map(c, b.LW, TX, TY, &a.mTw) ||
      (a.c2 && !make_compact_map(c, a.c2, TX + 8, TY + 6, &a.mC2)) || (a.grad && !make_compact_map(c, a.div, TX, TY, &a.mDiv)))
    return fail(SOLAR_ERR_CUDA, "cuTensorMapEncodeTiled failed");
  if (!a.c2) a.mC2 = a.mTq;                       // unused
  if (!a.grad) a.mDiv = a.mTq;
  static bool attr_set = false;
  static int resident = 1;
  if (!attr_set) {
    CK(cudaFuncSetAttribute(adj_stage_kernel<T, TX, TY>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::TOTAL));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, adj_stage_kernel<T, TX, TY>, TX * TY, L::TOTAL));
    resident = std::max(resident, 1);
    attr_set = true;
  }
  const Geom& g = c->g;
  // Radial chunks: the count that minimises waves x planes per CTA, a chunk reading three
  // planes more on either side (at 6 x 96^3 this picks 24-plane chunks, 2.92 waves: reverse
  // sweep 4.6% faster than 20-plane chunks in 3.65 waves, in both precisions).
  const long long tiles = 6LL * (g.n / TX) * (g.n / TY);
  const long long slots = (long long)c->nsm * resident;
  int best = 1;
  long long best_cost = -1;
  for (int nch = 1; nch <= std::max(1, g.nr / 8); ++nch) {
    const long long kc = (g.nr + nch - 1) / nch;
    const long long cost = ((tiles * nch + slots - 1) / slots) * (kc + 6);
    if (best_cost < 0 || cost < best_cost) { best_cost = cost; best = nch; }
  }
  a.kchunk = (g.nr + best - 1) / best;
  dim3 grid((unsigned)((g.n / TX) * (g.n / TY)), (unsigned)((g.nr + a.kchunk - 1) / a.kchunk), 6);
  adj_stage_kernel<T, TX, TY><<<grid, TX * TY, L::TOTAL, c->stream>>>(a);
  return SOLAR_OK;
}

template <typename T>
static int enqueue_rhs_adjoint(solar_ctx* c, AdjStageArgs<T> a) {
  AdjBuffers& b = c->adj;
  const Geom& g = c->g;
  a.lout = (T*)b.T1;
  a.lwout = (T*)b.T2;
  a.rb = (T*)b.rb;
  a.wc = wait_ctl(c, kInjAdjStage);
  if ((long long)g.nf * g.vs >= (1LL << 31))     // the kernel indexes one face's fields in 32 bits
    return fail(SOLAR_ERR_ARG, "grid too large for the adjoint (%lld values per face)", (long long)g.nf * g.vs);
  int rc = (g.n % 32 == 0) ? launch_adj_stage<T, 32, 8>(c, a) : launch_adj_stage<T, 16, 16>(c, a);
  if (rc) return rc;
  adj_rbdy_kernel<T><<<blocks_for(6LL * 14 * g.n * g.n, 256), 256, 0, c->stream>>>((T*)b.T1, (const T*)b.rb,
                                                                                   (const T*)c->dt.rad, g, a.dt);
  adj_edge_kernel<T><<<dim3(blocks_for(g.n, 128), 72, g.nr), 128, 2 * g.n * sizeof(T), c->stream>>>(
      (T*)b.T1, (const T*)b.wt, b.wt_span, b.tspan, g, 0);
  CK(cudaGetLastError());
  std::swap(b.L, b.T1);
  std::swap(b.LW, b.T2);
  return SOLAR_OK;
}

// FILTER_EXP^T in place on buffer L: radial^T, eta^T, xi^T, then the halo scatter.
template <typename T>
static int enqueue_filter_adjoint(solar_ctx* c) {
  const Geom& g = c->g;
  T* L = (T*)c->adj.L;
  T* T1 = (T*)c->adj.T1;
  adj_filter_r_kernel<T><<<blocks_for(6LL * g.nf * g.n * g.n, 128), 128, 0, c->stream>>>(L, T1, g);
  constexpr int KP = 8;                                             // planes per CTA
  const unsigned kch = (unsigned)((g.nr + KP - 1) / KP);
  constexpr int V = Vec16<T>::V;
  if (g.n % 32 == 0) {
    constexpr int TY = sizeof(T) == 4 ? 16 : 8;
    adj_filter_xyv_kernel<T, 32, TY><<<dim3((g.n / 32) * (g.n / TY), kch, 6 * g.nf), dim3(32 / V, TY), 0, c->stream>>>(
        T1, L, g, KP);
  } else {
    adj_filter_xyv_kernel<T, 16, 16><<<dim3((g.n / 16) * (g.n / 16), kch, 6 * g.nf), dim3(16 / V, 16), 0, c->stream>>>(
        T1, L, g, KP);
  }
  adj_edge_kernel<T><<<dim3(blocks_for(g.n, 128), 72, g.nr), 128, g.nf * g.n * sizeof(T), c->stream>>>(
      L, (const T*)c->adj.wt, c->adj.wt_span, c->adj.tspan, g, 1);
  CK(cudaGetLastError());
  return SOLAR_OK;
}

// One reverse time step on buffer L: lambda_n -> lambda_{n-1}.  `dstep` holds the
// divergence of the five stage inputs of the forward step (gradient only).
template <typename T>
static int enqueue_step_adjoint(solar_ctx* c, const T* dstep, double* grad) {
  int rc;
  if ((rc = enqueue_filter_adjoint<T>(c))) return rc;
  CK(cudaMemsetAsync(c->adj.LW, 0, (size_t)state_bytes(c), c->stream));
  const long long V6 = 6 * vol_compact(c);
  for (int s = 4; s >= 0; --s) {
    AdjStageArgs<T> a = adj_args<T>(c, c->desc.dt);
    a.alpha = s == 0 ? T(0) : (T)kAlpha[s];
    a.beta = (T)kBeta[s];
    a.keep = 1;
    if (grad && dstep) { a.grad = grad; a.div = dstep + s * V6; }
    if ((rc = enqueue_rhs_adjoint<T>(c, a))) return rc;
  }
  return SOLAR_OK;
}

// One forward step (same kernels as the step graph) that also stores the divergence of
// each stage input into dstep[stage][face][k][j][i].
template <typename T>
static int enqueue_step_div(solar_ctx* c, T* dstep) {
  void* bufs[2] = {c->A, c->B};
  const long long V6 = 6 * vol_compact(c);
  int cur = 0, rc;
  if ((rc = force_begin(c))) return rc;
  for (int s = 0; s < 5; ++s) {
    if ((rc = launch_edge<T>(c, bufs[cur], 0, nullptr))) return rc;
    if ((rc = launch_stage<T>(c, bufs[cur], bufs[cur ^ 1], s == 0 ? 4 : 5, s, nullptr, dstep + s * V6))) return rc;
    cur ^= 1;
  }
  if ((rc = launch_edge<T>(c, bufs[cur], 1, nullptr))) return rc;
  if ((rc = launch_filter<T>(c, bufs[cur], bufs[cur ^ 1], nullptr))) return rc;
  CK(cudaGetLastError());
  return force_end(c);
}

template <typename T>
static void enqueue_sample(solar_ctx* c, double* out) {
  const AdjBuffers& b = c->adj;
  sample_kernel<T><<<blocks_for(b.nrec, 128), 128, 0, c->stream>>>((const T*)c->A, b.rec_off, b.rec_w, b.nrec, out);
}

// The checkpointed sweep.  Outer checkpoints every K steps are kept for the whole run.  With
// K2 < K each outer segment is first run forward again keeping inner checkpoints every K2
// steps, and each inner segment is then recomputed storing its stage-input divergences and
// reversed; memory is one state per outer and per inner checkpoint plus 5 * K2 field volumes,
// for one more forward run than the single-level sweep (K2 = K).
template <typename T>
static int misfit_gradient_t(solar_ctx* c, int N, int K, int K2, const double* data, double* misfit, double* grad_c,
                             double* lambda0, double* times) {
  AdjBuffers& b = c->adj;
  const long long V6 = 6 * vol_compact(c);
  const size_t S = (size_t)state_bytes(c);
  const int ncp = (N + K - 1) / K;
  K2 = std::max(1, std::min(K2, K));
  const int nsub_max = (std::min(K, N) + K2 - 1) / K2;
  int rc;
  if ((rc = adj_reserve(&b.ckpt, &b.ckpt_bytes, S * (size_t)ncp))) return rc;
  if (nsub_max > 1 && (rc = adj_reserve(&b.ckpt2, &b.ckpt2_bytes, S * (size_t)nsub_max))) return rc;
  if ((rc = adj_reserve(&b.div, &b.div_bytes, (size_t)std::min(K2, N) * 5 * V6 * sizeof(T)))) return rc;
  if ((rc = adj_reserve((void**)&b.traces, &b.traces_bytes, (size_t)std::max(N, 1) * b.nrec * 2 * sizeof(double)))) return rc;
  // with a source term the clock (time, step, interpolation state) is checkpointed too
  const size_t CL = sizeof(ForceClock);
  if (c->forcing && (rc = adj_reserve(&b.clk, &b.clk_bytes, CL * (size_t)(ncp + nsub_max)))) return rc;
  char* clk = (char*)b.clk;
  char* clk2 = clk + CL * (size_t)ncp;
  char* ckpt2 = (char*)b.ckpt2;
  double* traces = b.traces;
  double* res = b.traces + (size_t)N * b.nrec;
  char* ckpt = (char*)b.ckpt;
  T* D = (T*)b.div;
  if ((rc = capture_step_graph(c))) return rc;
  CK(cudaEventRecord(c->ev[2], c->stream));
  // forward sweep: checkpoints every K steps, receiver traces after every step
  for (int n = 0; n < N; ++n) {
    if (n % K == 0) {
      CK(cudaMemcpyAsync(ckpt + (size_t)(n / K) * S, c->A, S, cudaMemcpyDeviceToDevice, c->stream));
      if (c->forcing) CK(cudaMemcpyAsync(clk + (size_t)(n / K) * CL, c->force_clock, CL, cudaMemcpyDeviceToDevice, c->stream));
    }
    CK(cudaGraphLaunch(c->step_graph, c->stream));
    enqueue_sample<T>(c, traces + (size_t)n * b.nrec);
  }
  CK(cudaEventRecord(c->ev[3], c->stream));
  std::vector<double> h((size_t)N * b.nrec);
  CK(cudaMemcpyAsync(h.data(), traces, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if ((rc = check_device_error(c))) return rc;
  double J = 0.0;
  for (size_t q = 0; q < h.size(); ++q) {
    h[q] -= data[q];
    J += 0.5 * h[q] * h[q];
  }
  if (misfit) *misfit = J;
  CK(cudaMemcpyAsync(res, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  // reverse sweep, one checkpoint segment at a time
  CK(cudaMemsetAsync(c->adj.L, 0, S, c->stream));
  CK(cudaMemsetAsync(b.grad, 0, (size_t)V6 * sizeof(double), c->stream));
  float t_rec = 0.f, t_adj = 0.f;
  for (int seg = ncp - 1; seg >= 0; --seg) {
    const int n0 = seg * K, n1 = std::min(N, n0 + K);
    const int nsub = (n1 - n0 + K2 - 1) / K2;
    CK(cudaEventRecord(c->ev[4], c->stream));
    CK(cudaMemcpyAsync(c->A, ckpt + (size_t)seg * S, S, cudaMemcpyDeviceToDevice, c->stream));
    if (c->forcing) CK(cudaMemcpyAsync(c->force_clock, clk + (size_t)seg * CL, CL, cudaMemcpyDeviceToDevice, c->stream));
    if (nsub > 1)                  // inner checkpoints of this segment
      for (int n = n0; n < n1; ++n) {
        if ((n - n0) % K2 == 0) {
          const size_t q = (size_t)((n - n0) / K2);
          CK(cudaMemcpyAsync(ckpt2 + q * S, c->A, S, cudaMemcpyDeviceToDevice, c->stream));
          if (c->forcing) CK(cudaMemcpyAsync(clk2 + q * CL, c->force_clock, CL, cudaMemcpyDeviceToDevice, c->stream));
        }
        CK(cudaGraphLaunch(c->step_graph, c->stream));
      }
    CK(cudaEventRecord(c->ev[7], c->stream));
    CK(cudaEventSynchronize(c->ev[7]));
    float r0 = 0.f;
    CK(cudaEventElapsedTime(&r0, c->ev[4], c->ev[7]));
    t_rec += r0;
    for (int sub = nsub - 1; sub >= 0; --sub) {
      const int m0 = n0 + sub * K2, m1 = std::min(n1, m0 + K2);
      CK(cudaEventRecord(c->ev[4], c->stream));
      if (nsub > 1) {
        CK(cudaMemcpyAsync(c->A, ckpt2 + (size_t)sub * S, S, cudaMemcpyDeviceToDevice, c->stream));
        if (c->forcing) CK(cudaMemcpyAsync(c->force_clock, clk2 + (size_t)sub * CL, CL, cudaMemcpyDeviceToDevice, c->stream));
      }
      for (int n = m0; n < m1; ++n)
        if ((rc = enqueue_step_div<T>(c, D + (size_t)(n - m0) * 5 * V6))) return rc;
      CK(cudaEventRecord(c->ev[5], c->stream));
      for (int n = m1; n > m0; --n) {
        // lambda += S^T (S q_n - d_n), then lambda <- STEP^T lambda (with the gradient)
        inject_kernel<T><<<blocks_for(b.nrec, 128), 128, 0, c->stream>>>((T*)c->adj.L, b.rec_off, b.rec_w, b.nrec,
                                                                          res + (size_t)(n - 1) * b.nrec);
        if ((rc = enqueue_step_adjoint<T>(c, D + (size_t)(n - 1 - m0) * 5 * V6, b.grad))) return rc;
      }
      CK(cudaEventRecord(c->ev[6], c->stream));
      CK(cudaEventSynchronize(c->ev[6]));
      float a = 0.f, r = 0.f;
      CK(cudaEventElapsedTime(&r, c->ev[4], c->ev[5]));
      CK(cudaEventElapsedTime(&a, c->ev[5], c->ev[6]));
      t_rec += r;
      t_adj += a;
    }
  }
  // leave the state (and the clock) at the initial condition
  CK(cudaMemcpyAsync(c->A, ckpt, S, cudaMemcpyDeviceToDevice, c->stream));
  if (c->forcing) CK(cudaMemcpyAsync(c->force_clock, clk, CL, cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if ((rc = check_device_error(c))) return rc;
  if (times) {
    float f = 0.f;
    CK(cudaEventElapsedTime(&f, c->ev[2], c->ev[3]));
    times[0] = f;
    times[1] = t_rec;
    times[2] = t_adj;
  }
  if (grad_c) {
    CK(cudaMemcpyAsync(grad_c, b.grad, (size_t)V6 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
  if (lambda0) return download_fields(c, c->adj.L, 0, lambda0, 5, kAllFields, 5);
  return SOLAR_OK;
}

}  // namespace solar

extern "C" {

int solar_gpu_set_receivers(solar_ctx* c, int nrec, const double* loc) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (nrec < 1 || !loc) return fail(SOLAR_ERR_ARG, "need nrec >= 1 and receiver locations");
  if ((rc = adj_alloc(c))) return rc;
  const Geom& g = c->g;
  std::vector<long long> off((size_t)nrec * 8);
  std::vector<double> w((size_t)nrec * 8);
  for (int r = 0; r < nrec; ++r) {
    const double f = loc[r * 4 + 0], x = loc[r * 4 + 1], y = loc[r * 4 + 2], z = loc[r * 4 + 3];
    const int face = (int)f;
    if (face != f || face < 0 || face > 5 || !(x >= 0 && x <= g.n - 1) || !(y >= 0 && y <= g.n - 1) ||
        !(z >= 0 && z <= g.nr - 1))
      return fail(SOLAR_ERR_ARG, "receiver %d outside the grid (face %g, i %g, j %g, k %g)", r, f, x, y, z);
    const int i0 = std::min((int)x, g.n - 2), j0 = std::min((int)y, g.n - 2), k0 = std::min((int)z, g.nr - 2);
    const double wx = x - i0, wy = y - j0, wz = z - k0;
    for (int cc = 0; cc < 8; ++cc) {
      const int di = cc & 1, dj = (cc >> 1) & 1, dk = cc >> 2;
      off[(size_t)r * 8 + cc] = g.vol(0, face, g.slot[kP]) + g.at(k0 + dk, j0 + dj, i0 + di);
      w[(size_t)r * 8 + cc] = (di ? wx : 1 - wx) * (dj ? wy : 1 - wy) * (dk ? wz : 1 - wz);
    }
  }
  AdjBuffers& b = c->adj;
  if (b.rec_off) cudaFree(b.rec_off);
  if (b.rec_w) cudaFree(b.rec_w);
  b.rec_off = nullptr;
  b.rec_w = nullptr;
  b.nrec = 0;
  CK(cudaMalloc((void**)&b.rec_off, off.size() * sizeof(long long)));
  CK(cudaMalloc((void**)&b.rec_w, w.size() * sizeof(double)));
  CK(cudaMemcpy(b.rec_off, off.data(), off.size() * sizeof(long long), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(b.rec_w, w.data(), w.size() * sizeof(double), cudaMemcpyHostToDevice));
  b.nrec = nrec;
  return SOLAR_OK;
}

int solar_gpu_record(solar_ctx* c, int nsteps, double* traces) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (nsteps < 0 || !traces) return fail(SOLAR_ERR_ARG, "bad arguments");
  if (!c->adj.nrec) return fail(SOLAR_ERR_STATE, "no receivers set");
  AdjBuffers& b = c->adj;
  if ((rc = adj_reserve((void**)&b.traces, &b.traces_bytes, (size_t)std::max(nsteps, 1) * b.nrec * 2 * sizeof(double))))
    return rc;
  if ((rc = capture_step_graph(c))) return rc;
  for (int n = 0; n < nsteps; ++n) {
    CK(cudaGraphLaunch(c->step_graph, c->stream));
    if (c->fp32) enqueue_sample<float>(c, b.traces + (size_t)n * b.nrec);
    else enqueue_sample<double>(c, b.traces + (size_t)n * b.nrec);
  }
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(traces, b.traces, (size_t)nsteps * b.nrec * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return check_device_error(c);
}

int solar_gpu_misfit_gradient(solar_ctx* c, int nsteps, int checkpoint_every, const double* data,
                              double* misfit, double* grad_c, double* lambda0, double* times_ms) {
  return solar_gpu_misfit_gradient_nested(c, nsteps, checkpoint_every, checkpoint_every, data, misfit, grad_c,
                                          lambda0, times_ms);
}

int solar_gpu_misfit_gradient_nested(solar_ctx* c, int nsteps, int checkpoint_every, int inner_every,
                                     const double* data, double* misfit, double* grad_c, double* lambda0,
                                     double* times_ms) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (inner_every < 1) return fail(SOLAR_ERR_ARG, "need inner_every >= 1");
  if (nsteps < 1 || checkpoint_every < 1 || !data) return fail(SOLAR_ERR_ARG, "need nsteps >= 1, checkpoint_every >= 1 and data");
  if (!c->adj.nrec) return fail(SOLAR_ERR_STATE, "no receivers set");
  if ((rc = adj_alloc(c))) return rc;
  return c->fp32 ? misfit_gradient_t<float>(c, nsteps, checkpoint_every, inner_every, data, misfit, grad_c, lambda0, times_ms)
                 : misfit_gradient_t<double>(c, nsteps, checkpoint_every, inner_every, data, misfit, grad_c, lambda0, times_ms);
}

int solar_gpu_rhs_adjoint(solar_ctx* c, const double* mu, double* out) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!mu || !out) return fail(SOLAR_ERR_ARG, "null array");
  if ((rc = adj_alloc(c))) return rc;
  if ((rc = upload_fields(c, c->adj.L, 0, mu, 5, kAllFields, 5))) return rc;
  CK(cudaMemsetAsync(c->adj.LW, 0, (size_t)state_bytes(c), c->stream));
  rc = c->fp32 ? enqueue_rhs_adjoint<float>(c, adj_args<float>(c, 1.0))
               : enqueue_rhs_adjoint<double>(c, adj_args<double>(c, 1.0));
  if (rc) return rc;
  if ((rc = download_fields(c, c->adj.L, 0, out, 5, kAllFields, 5))) return rc;
  return check_device_error(c);
}

int solar_gpu_filter_adjoint(solar_ctx* c, const double* lam, double* out) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!lam || !out) return fail(SOLAR_ERR_ARG, "null array");
  if ((rc = adj_alloc(c))) return rc;
  if ((rc = upload_fields(c, c->adj.L, 0, lam, 5, kAllFields, 5))) return rc;
  rc = c->fp32 ? enqueue_filter_adjoint<float>(c) : enqueue_filter_adjoint<double>(c);
  if (rc) return rc;
  if ((rc = download_fields(c, c->adj.L, 0, out, 5, kAllFields, 5))) return rc;
  return check_device_error(c);
}

int solar_gpu_rk4_adjoint(solar_ctx* c, int nsteps, const double* lam_in, double* lam_out) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (nsteps < 0 || !lam_in || !lam_out) return fail(SOLAR_ERR_ARG, "bad arguments");
  if ((rc = adj_alloc(c))) return rc;
  CK(cudaMemsetAsync(c->adj.L, 0, (size_t)state_bytes(c), c->stream));
  if ((rc = upload_fields(c, c->adj.L, 0, lam_in, 5, kAllFields, 5))) return rc;
  for (int n = 0; n < nsteps; ++n) {
    rc = c->fp32 ? enqueue_step_adjoint<float>(c, nullptr, nullptr) : enqueue_step_adjoint<double>(c, nullptr, nullptr);
    if (rc) return rc;
  }
  if ((rc = download_fields(c, c->adj.L, 0, lam_out, 5, kAllFields, 5))) return rc;
  return check_device_error(c);
}

}  // extern "C"
