// forcing.cuh -- the v_r source term of COMPUTE_RHS, on the device.  Included once, by
// solar_gpu.cu, after the context definition.
//
//   SOLAR_FORCING_ANALYTIC  compute_rhs_acoustic.f90:92-104: S = mag(t) exp(-((theta-pi/2)/
//       (20 dxi))^2 - (phi/(20 dxi))^2 - ((r - r_c)/(20 dchi))^2), mag(t) = exp(-(tau-650)^2 /
//       (2 200^2)) cos(4 pi (tau-650)/700), tau = t diml/dimc.  The reference fixes r_c at
//       gr(200); here the centre plane is a parameter.
//   SOLAR_FORCING_SAMPLES   LAGRANGE_INTERP (interpolation.f90:385-451) of the sampled
//       S_t(x, y, n) of READ_FORCING_FUNC (output.f90:271-307), added at plane e_rad
//       (compute_rhs_acoustic.f90:107-116, commented out in the reference).
// Every stage of one RK4 call sees the time of the call (time advances after FILTER_EXP,
// timestep.f90:82).  A one-thread clock kernel at the start of each step evaluates the
// time factors (including the reference's coefficient refresh when floor(xt) advances),
// a field kernel forms this step's S(x, y) for all faces, the stage kernel adds S(x, y)
// times the radial factor to the v_r right-hand side, and a clock kernel after the filter
// advances time and step.
#pragma once

namespace solar {

struct ForceClock {
  double time;          // COMMON /TSTEP/ time
  int step;             // the driver's step counter (cube.f90:71)
  int step_old;         // COMMON /STEP_TRACK/ (interpolation.f90:399)
  double x[7];          // COMMON /TIME_INTERP/ nodes
  double den[7];        // Lagrange denominators of the nodes
  int idx[7];           // 0-based sample of each node, -1 if that coefficient is zero
  double d[7];          // xt - x_m at this step's evaluation time
  double mag;           // analytic magnitude at this step
};

__global__ void force_clock_kernel(ForceClock* c, int kind, double diml, double dimc, double dt, double cad, int nstep,
                                   int nt, int* err) {
  if (threadIdx.x || blockIdx.x) return;
  if (kind == SOLAR_FORCING_ANALYTIC) {
    const double u = c->time * diml / dimc - 650.0;
    c->mag = exp(-(u * u) / (2.0 * 200.0 * 200.0)) * cos(4.0 * acos(-1.0) * u / 700.0);
    return;
  }
  double xt = (double)c->step * dt / cad + 1.0;
  const int fl = (int)floor(xt);
  if (c->step_old < fl) {
    for (int m = 0; m < 7; ++m) c->x[m] = (xt - (double)(4 - m)) * cad;
    for (int m = 0; m < 7; ++m) {
      double p = 1.0;
      bool first = true;
      for (int j = 0; j < 7; ++j) {
        if (j == m) continue;
        p = first ? (c->x[m] - c->x[j]) : p * (c->x[m] - c->x[j]);
        first = false;
      }
      c->den[m] = p;
      bool on = m >= 4 ? (m == 4 || (m == 5 && fl < nstep) || (m == 6 && fl < nstep - 1)) : c->x[m] >= 0.0;
      int s = fl - 4 + m;                        // S_t(:,:,floor(xt)-3+m), 1-based
      if (on && (s < 0 || s >= nt)) { on = false; atomicExch(err, kErrForcingSample); }
      c->idx[m] = on ? s : -1;
    }
    c->step_old = fl;
  }
  xt = ((double)c->step - 1.0) * dt;
  for (int m = 0; m < 7; ++m) c->d[m] = xt - c->x[m];
}

template <typename T>
__global__ void force_field_kernel(const ForceClock* c, int kind, const double* exy, const double* samples,
                                   long long n6, T* out) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n6) return;
  if (kind == SOLAR_FORCING_ANALYTIC) {
    out[p] = (T)(c->mag * exy[p]);
    return;
  }
  // forcing = LC0 (xt-x1)...(xt-x6) + LC1 (xt-x0)(xt-x2)... + ..., LC_m = S_t(idx_m) / den_m
  double f = 0.0;
  bool any = false;
  for (int m = 0; m < 7; ++m) {
    if (c->idx[m] < 0) continue;
    double t = samples[(long long)c->idx[m] * n6 + p] / c->den[m];
    for (int j = 0; j < 7; ++j)
      if (j != m) t = t * c->d[j];
    f = any ? f + t : t;
    any = true;
  }
  out[p] = (T)f;
}

__global__ void force_advance_kernel(ForceClock* c, double dt) {
  if (threadIdx.x || blockIdx.x) return;
  c->time = c->time + dt;
  c->step = c->step + 1;
}

// Nearest plane to r (ties to the outer plane), as SOLAR_DATA picks e_rad and o_rad.
static int nearest_plane(const solar_ctx* c, double r) {
  double temp = 1.0;
  int o = 0;
  for (int k = 0; k < c->g.nr; ++k)
    if (std::fabs(c->ht.gr[k] - r) <= temp) {
      temp = std::fabs(c->ht.gr[k] - r);
      o = k;
    }
  return o;
}

static int force_begin(solar_ctx* c) {
  if (!c->forcing) return SOLAR_OK;
  force_clock_kernel<<<1, 1, 0, c->stream>>>((ForceClock*)c->force_clock, c->forcing, 695.9894e8, c->ht.dimc,
                                             c->desc.dt, c->force_cad, c->force_nstep, c->force_nt, c->err);
  const long long n6 = 6LL * c->g.n * c->g.n;
  const unsigned blocks = (unsigned)((n6 + 255) / 256);
  if (c->fp32)
    force_field_kernel<float><<<blocks, 256, 0, c->stream>>>((const ForceClock*)c->force_clock, c->forcing,
                                                             c->force_exy, c->force_samples, n6, (float*)c->force_xy);
  else
    force_field_kernel<double><<<blocks, 256, 0, c->stream>>>((const ForceClock*)c->force_clock, c->forcing,
                                                              c->force_exy, c->force_samples, n6, (double*)c->force_xy);
  CK(cudaGetLastError());
  return SOLAR_OK;
}

static int force_end(solar_ctx* c) {
  if (!c->forcing) return SOLAR_OK;
  force_advance_kernel<<<1, 1, 0, c->stream>>>((ForceClock*)c->force_clock, c->desc.dt);
  CK(cudaGetLastError());
  return SOLAR_OK;
}

template <typename T>
static int upload_as(void* dst, const std::vector<double>& v) {
  std::vector<T> t(v.begin(), v.end());
  CK(cudaMemcpy(dst, t.data(), t.size() * sizeof(T), cudaMemcpyHostToDevice));
  return SOLAR_OK;
}

}  // namespace solar

extern "C" {

int solar_gpu_set_forcing(solar_ctx* c, int kind, int k_center, int nstep) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (kind < SOLAR_FORCING_OFF || kind > SOLAR_FORCING_SAMPLES) return fail(SOLAR_ERR_ARG, "unknown forcing kind %d", kind);
  if (kind != SOLAR_FORCING_OFF && c->g.nruns != 1) return fail(SOLAR_ERR_ARG, "forcing needs nruns == 1");
  if (kind == SOLAR_FORCING_ANALYTIC && (k_center < 0 || k_center >= c->g.nr))
    return fail(SOLAR_ERR_ARG, "forcing centre plane %d outside 0..%d", k_center, c->g.nr - 1);
  if (kind == SOLAR_FORCING_SAMPLES && !c->force_samples)
    return fail(SOLAR_ERR_STATE, "set the forcing samples of all six zones first");
  CK(cudaStreamSynchronize(c->stream));
  const int n = c->g.n, nr = c->g.nr;
  const size_t n6 = (size_t)6 * n * n;
  if (!c->force_clock) {
    CK(cudaMalloc(&c->force_clock, sizeof(ForceClock)));
    CK(cudaMemset(c->force_clock, 0, sizeof(ForceClock)));
    CK(cudaMalloc(&c->force_xy, n6 * c->esize));
    CK(cudaMalloc(&c->force_r, (size_t)nr * c->esize));
  }
  const double dimc = c->ht.dimc;                      // model row 1 sound speed (SOLAR_DATA)
  const double diml = 695.9894e8;                      // rsun (ic_acoustic_wave.f90:76)
  c->force_cad = 60.0 * dimc / diml;                   // cadforcing (ic_acoustic_wave.f90:113)
  c->force_nstep = nstep;
  std::vector<double> fr((size_t)nr, 0.0);
  if (kind == SOLAR_FORCING_ANALYTIC) {
    if (!c->force_exy) {
      // theta, phi of SETUP_COORDINATES_METRICS_ALL (metric.f90:95-158)
      const double pi = std::acos(-1.0), w = 20.0 * c->ht.dxi;
      std::vector<double> e(n6);
      for (int z = 0; z < 6; ++z)
        for (int j = 0; j < n; ++j)
          for (int i = 0; i < n; ++i) {
            const double xi = c->ht.gxi[i], tx = c->ht.tanx[i], ty = c->ht.tanx[j];
            double th, ph;
            if (z == 0) { ph = xi; th = std::atan(1.0 / (ty * std::cos(ph))); }
            else if (z == 1) { ph = xi + pi * 0.5; th = std::atan(1.0 / (ty * std::sin(ph))); }
            else if (z == 2) { ph = xi + pi; th = std::atan(-1.0 / (ty * std::cos(ph))); }
            else if (z == 3) { ph = xi + pi * 1.5; th = std::atan(-1.0 / (ty * std::sin(ph))); }
            else if (z == 4) { th = std::atan(std::sqrt(tx * tx + ty * ty)); ph = std::atan2(tx, -ty); }
            else { th = pi - std::atan(std::sqrt(tx * tx + ty * ty)); ph = std::atan2(tx, ty); }
            if (z <= 3 && th < 0) th += pi;
            if (z >= 1 && ph < 0) ph += 2.0 * pi;
            const double a = (th - pi / 2.0) / w, b = (ph - 0.0) / w;
            e[((size_t)z * n + j) * n + i] = std::exp(-(a * a) - b * b);
          }
      CK(cudaMalloc((void**)&c->force_exy, n6 * sizeof(double)));
      CK(cudaMemcpy(c->force_exy, e.data(), n6 * sizeof(double), cudaMemcpyHostToDevice));
    }
    const double wr = 20.0 * c->ht.dchi;
    for (int k = 0; k < nr; ++k) {
      const double u = (c->ht.gr[k] - c->ht.gr[k_center]) / wr;
      fr[k] = std::exp(-(u * u));
    }
  } else if (kind == SOLAR_FORCING_SAMPLES) {
    fr[nearest_plane(c, 1.0 - 100e5 / diml)] = 1.0;   // e_rad (ic_acoustic_wave.f90:117-122)
  }
  if (kind != SOLAR_FORCING_OFF) {
    rc = c->fp32 ? upload_as<float>(c->force_r, fr) : upload_as<double>(c->force_r, fr);
    if (rc) return rc;
  }
  c->forcing = kind;
  if (c->step_graph) { cudaGraphExecDestroy(c->step_graph); c->step_graph = nullptr; }
  drop_batch_graphs(c);
  return SOLAR_OK;
}

int solar_gpu_set_forcing_samples(solar_ctx* c, int zone, const double* f, int nt) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!f || zone < 0 || zone > 5 || nt < 1) return fail(SOLAR_ERR_ARG, "bad zone, samples or nt");
  if (c->force_samples && nt != c->force_nt) return fail(SOLAR_ERR_ARG, "nt differs from the other zones' (%d)", c->force_nt);
  const int n = c->g.n;
  const size_t n6 = (size_t)6 * n * n;
  if (!c->force_samples) {
    CK(cudaMalloc((void**)&c->force_samples, (size_t)nt * n6 * sizeof(double)));
    CK(cudaMemset(c->force_samples, 0, (size_t)nt * n6 * sizeof(double)));
    c->force_nt = nt;
  }
  // READ_FORCING_FUNC order: f(i, j, n) with n fastest, then j, then i -> [n][zone][j][i]
  std::vector<double> t((size_t)nt * n * n);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j)
      for (int m = 0; m < nt; ++m) t[((size_t)m * n + j) * n + i] = f[((size_t)i * n + j) * nt + m];
  for (int m = 0; m < nt; ++m)
    CK(cudaMemcpy(c->force_samples + (size_t)m * n6 + (size_t)zone * n * n, t.data() + (size_t)m * n * n,
                  (size_t)n * n * sizeof(double), cudaMemcpyHostToDevice));
  return SOLAR_OK;
}

int solar_gpu_set_clock(solar_ctx* c, double time, int step) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!c->force_clock) {
    CK(cudaMalloc(&c->force_clock, sizeof(ForceClock)));
    const size_t n6 = (size_t)6 * c->g.n * c->g.n;
    CK(cudaMalloc(&c->force_xy, n6 * c->esize));
    CK(cudaMalloc(&c->force_r, (size_t)c->g.nr * c->esize));
  }
  ForceClock h;
  std::memset(&h, 0, sizeof h);
  h.time = time;
  h.step = step;
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaMemcpy(c->force_clock, &h, sizeof h, cudaMemcpyHostToDevice));
  return SOLAR_OK;
}

int solar_gpu_get_clock(solar_ctx* c, double* time, int* step) {
  int rc = check_ctx(c);
  if (rc) return rc;
  ForceClock h;
  std::memset(&h, 0, sizeof h);
  if (c->force_clock) {
    CK(cudaStreamSynchronize(c->stream));
    CK(cudaMemcpy(&h, c->force_clock, sizeof h, cudaMemcpyDeviceToHost));
  }
  if (time) *time = h.time;
  if (step) *step = h.step;
  return SOLAR_OK;
}

}  // extern "C"
