// io_host.cuh -- context-level writers/readers of the reference's output files: the data
// each file needs (one plane, one column, or the whole state) is gathered on the device and
// written by the host functions of io.cpp.  Included once, by solar_gpu.cu.
#pragma once

extern "C" {
int solar_io_cue_name(int cue, char* buf, int len);
int solar_io_write_restart(const char* path, const double* q, int nx, int ny, int nr, double time, int step);
int solar_io_read_restart(const char* path, double* q, int nx, int ny, int nr, double* time, int* step);
int solar_io_write_visual(const char* path, const double* plane5, int nx, int ny);
int solar_io_write_grid(const char* path, const int* seven);
int solar_io_append_trace(const char* path, const double* values, int count);
int solar_io_read_forcing(const char* path, int nx, int ny, int nt, double* f);
int solar_gpu_set_forcing_samples(solar_ctx* c, int zone, const double* f, int nt);
}

namespace solar {

// out[zone][field][j][i] = q at plane k (FP64), reference field order, absent rho -> 0
template <typename T>
__global__ void gather_plane_kernel(const T* q, double* out, Geom g, int run, int k) {
  const long long P2 = (long long)g.n * g.n;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= 30 * P2) return;
  const int zf = (int)(idx / P2), p2 = (int)(idx % P2);
  const int z = zf / 5, f = zf % 5, s = g.slot[f];
  out[idx] = s < 0 ? 0.0 : (double)q[g.vol(run, z, s) + g.at(k, p2 / g.n, p2 % g.n)];
}

// out[zone][field][k] = q at column (i, j)
template <typename T>
__global__ void gather_column_kernel(const T* q, double* out, Geom g, int run, int i, int j) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= 30 * g.nr) return;
  const int zf = idx / g.nr, k = idx % g.nr;
  const int z = zf / 5, f = zf % 5, s = g.slot[f];
  out[idx] = s < 0 ? 0.0 : (double)q[g.vol(run, z, s) + g.at(k, j, i)];
}

// o_rad of SOLAR_DATA (ic_acoustic_wave.f90:124-132): the plane nearest r = 1 + 200 km / R_sun,
// ties to the outer plane; 0-based.
static int output_plane(const solar_ctx* c) {
  const double obsheight = 1.0 + 200e5 / 695.9894e8;
  double temp = 1.0;
  int o = c->g.nr - 1;
  for (int k = 0; k < c->g.nr; ++k)
    if (std::fabs(c->ht.gr[k] - obsheight) <= temp) {
      temp = std::fabs(c->ht.gr[k] - obsheight);
      o = k;
    }
  return o;
}

static std::string cue_str(int cue) {
  char b[32];
  solar_io_cue_name(cue, b, sizeof b);
  return b;
}

static int gather_small(solar_ctx* c, int run, bool plane, int a0, int a1, std::vector<double>& host) {
  const long long n = plane ? 30LL * c->g.n * c->g.n : 30LL * c->g.nr;
  double* d = nullptr;
  CK(cudaMalloc((void**)&d, (size_t)n * sizeof(double)));
  const unsigned blocks = (unsigned)((n + 255) / 256);
  if (plane) {
    if (c->fp32) gather_plane_kernel<float><<<blocks, 256, 0, c->stream>>>((const float*)c->A, d, c->g, run, a0);
    else gather_plane_kernel<double><<<blocks, 256, 0, c->stream>>>((const double*)c->A, d, c->g, run, a0);
  } else {
    if (c->fp32) gather_column_kernel<float><<<blocks, 256, 0, c->stream>>>((const float*)c->A, d, c->g, run, a0, a1);
    else gather_column_kernel<double><<<blocks, 256, 0, c->stream>>>((const double*)c->A, d, c->g, run, a0, a1);
  }
  host.resize((size_t)n);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(host.data(), d, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(d);
  if (e != cudaSuccess) return fail(SOLAR_ERR_CUDA, "output gather: %s", cudaGetErrorString(e));
  return SOLAR_OK;
}

static int check_out_args(solar_ctx* c, int run, const char* dir) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!dir || run < 0 || run >= c->g.nruns) return fail(SOLAR_ERR_ARG, "bad run or null directory");
  return SOLAR_OK;
}

}  // namespace solar

extern "C" {

int solar_gpu_output_plane(solar_ctx* c, int* k) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!k) return fail(SOLAR_ERR_ARG, "null output");
  *k = output_plane(c);
  return SOLAR_OK;
}

int solar_gpu_write_visual(solar_ctx* c, int run, const char* dir, int cue) {
  int rc = check_out_args(c, run, dir);
  if (rc) return rc;
  if (cue < 0) return fail(SOLAR_ERR_ARG, "cue < 0");
  std::vector<double> h;
  if ((rc = gather_small(c, run, true, output_plane(c), 0, h))) return rc;
  const size_t per = (size_t)5 * c->g.n * c->g.n;
  for (int z = 0; z < 6; ++z) {
    const std::string path = std::string(dir) + "/Visual/" + cue_str(cue) + "/vis_" + std::to_string(z);
    if ((rc = solar_io_write_visual(path.c_str(), h.data() + z * per, c->g.n, c->g.n))) return rc;
  }
  return SOLAR_OK;
}

int solar_gpu_write_grid(solar_ctx* c, const char* dir) {
  int rc = check_out_args(c, 0, dir);
  if (rc) return rc;
  for (int z = 0; z < 6; ++z) {
    const int seven[7] = {0, c->g.n - 1, 0, c->g.n - 1, 0, c->g.nr - 1, z + 1};
    const std::string path = std::string(dir) + "/Visual/grid/grid_" + std::to_string(z);
    if ((rc = solar_io_write_grid(path.c_str(), seven))) return rc;
  }
  return SOLAR_OK;
}

int solar_gpu_write_radial_trace(solar_ctx* c, int run, const char* dir) {
  int rc = check_out_args(c, run, dir);
  if (rc) return rc;
  std::vector<double> h;
  if ((rc = gather_small(c, run, false, 0, 0, h))) return rc;
  const size_t per = (size_t)5 * c->g.nr;
  for (int z = 0; z < 6; ++z) {
    const std::string path = std::string(dir) + "/trace_" + std::to_string(z + 1);
    if ((rc = solar_io_append_trace(path.c_str(), h.data() + z * per, (int)per))) return rc;
  }
  return SOLAR_OK;
}

int solar_gpu_load_forcing(solar_ctx* c, const char* dir, int nt) {
  int rc = check_out_args(c, 0, dir);
  if (rc) return rc;
  if (nt < 1) return fail(SOLAR_ERR_ARG, "nt < 1");
  std::vector<double> f((size_t)c->g.n * c->g.n * nt);
  for (int z = 0; z < 6; ++z) {
    const std::string path = std::string(dir) + "/forcing/forcing_cubesph." + std::to_string(z + 1);
    if ((rc = solar_io_read_forcing(path.c_str(), c->g.n, c->g.n, nt, f.data()))) return rc;
    if ((rc = solar_gpu_set_forcing_samples(c, z, f.data(), nt))) return rc;
  }
  return SOLAR_OK;
}

int solar_gpu_write_restart(solar_ctx* c, int run, const char* dir, int cue, double time, int step) {
  int rc = check_out_args(c, run, dir);
  if (rc) return rc;
  if (cue < 0) return fail(SOLAR_ERR_ARG, "cue < 0");
  const long long V = vol_compact(c);
  std::vector<double> q((size_t)30 * V);
  if ((rc = download_fields(c, c->A, run, q.data(), 5, kAllFields, 5))) return rc;
  for (int z = 0; z < 6; ++z) {
    const std::string path = std::string(dir) + "/Restart/restart." + cue_str(cue) + "." + std::to_string(z + 1);
    if ((rc = solar_io_write_restart(path.c_str(), q.data() + (size_t)z * 5 * V, c->g.n, c->g.n, c->g.nr, time, step)))
      return rc;
  }
  return SOLAR_OK;
}

int solar_gpu_read_restart(solar_ctx* c, int run, const char* dir, int cue, double* time, int* step) {
  int rc = check_out_args(c, run, dir);
  if (rc) return rc;
  if (cue < 0) return fail(SOLAR_ERR_ARG, "cue < 0");
  const long long V = vol_compact(c);
  std::vector<double> q((size_t)30 * V);
  double t0 = 0;
  int s0 = 0;
  for (int z = 0; z < 6; ++z) {
    const std::string path = std::string(dir) + "/Restart/restart." + cue_str(cue) + "." + std::to_string(z + 1);
    double t = 0;
    int s = 0;
    if ((rc = solar_io_read_restart(path.c_str(), q.data() + (size_t)z * 5 * V, c->g.n, c->g.n, c->g.nr, &t, &s)))
      return rc;
    if (z == 0) { t0 = t; s0 = s; }
    else if (t != t0 || s != s0) return fail(SOLAR_ERR_ARG, "restart files of cue %d disagree on time/step", cue);
  }
  if ((rc = upload_fields(c, c->A, run, q.data(), 5, kAllFields, 5))) return rc;
  CK(cudaStreamSynchronize(c->stream));
  if (time) *time = t0;
  if (step) *step = s0;
  return SOLAR_OK;
}

}  // extern "C"
