// curl.cuh -- COMPUTE_CURL (grad.f90:140-255) on the device: the halo exchange of a_r
// (scalar) and of (a_xi, a_eta) with both receiver-frame components
// (TRANSFORM_VECTOR_BETWEEN_MESHES_CURL, transform.f90:279-498, folded into one coefficient
// set per ghost point and tap), then the DRP derivatives and the curl formula of
// grad.f90:233-244 per point.  An operator-level entry point, not on the time-stepping
// path.  Included once, by solar_gpu.cu.
#pragma once

namespace solar {

// Ghost frames of a_r (v_r slot, scalar) and (a_xi, a_eta) (v_xi, v_eta slots, both
// components) of run 0.  grid: x over positions t, y over (receiving face-edge, layer), z over planes.
template <typename T>
__global__ void curl_edge_kernel(T* q, const T* __restrict__ ew, const T* __restrict__ egc, const int* __restrict__ s0t,
                                 Geom g) {
  const int n = g.n;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int fe = blockIdx.y / 3, l = blockIdx.y % 3, k = blockIdx.z;
  const int face = fe >> 2, e = fe & 3;
  const EdgeRouteDev rt = cRoute[face][e];
  const bool along_i = rt.src_edge <= 1;
  const int fixed = (rt.src_edge == 0 || rt.src_edge == 2) ? l + 1 : n - 2 - l;
  const int crow = (fe * 3 + l) * 9;
  const int s0 = s0t[(fe * 3 + l) * n + t];
  long long dst;
  if (e == 0) dst = g.at(k, -1 - l, t);
  else if (e == 1) dst = g.at(k, n + l, t);
  else if (e == 2) dst = g.at(k, t, -1 - l);
  else dst = g.at(k, t, n + l);
  const T* sr = q + g.vol(0, rt.src_face, g.slot[kVr]);
  const T* sx = q + g.vol(0, rt.src_face, g.slot[kVxi]);
  const T* sy = q + g.vol(0, rt.src_face, g.slot[kVeta]);
  T gr = T(0), gx = T(0), gy = T(0);
  for (int s = 0; s < 9; ++s) {
    const int ii = along_i ? s0 + s : fixed, jj = along_i ? fixed : s0 + s;
    const long long o = g.at(k, jj, ii);
    const T vx = sx[o], vy = sy[o];
    const T* c = egc + ((long long)(crow + s) * 4) * n + t;   // [out][in] with stride n
    gr += ew[(long long)(crow + s) * n + t] * sr[o];
    gx += c[0] * vx + c[n] * vy;
    gy += c[2 * n] * vx + c[3 * n] * vy;
  }
  q[g.vol(0, face, g.slot[kVr]) + dst] = gr;
  q[g.vol(0, face, g.slot[kVxi]) + dst] = gx;
  q[g.vol(0, face, g.slot[kVeta]) + dst] = gy;
}

// curl_xi, curl_eta, curl_r (grad.f90:233-244) into the v_xi, v_eta, v_r slots of `out`.
template <typename T>
__global__ void curl_kernel(const T* q, T* out, const double* __restrict__ tanx, const double* __restrict__ gr,
                            const T* __restrict__ rad, Geom g, double inv_dxi) {
  const int n = g.n, nr = g.nr;
  const long long V = (long long)n * n * nr;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= 6 * V) return;
  const int face = (int)(idx / V);
  const long long l = idx % V;
  const int i = (int)(l % n), j = (int)((l / n) % n), k = (int)(l / ((long long)n * n));
  const T* ax = q + g.vol(0, face, g.slot[kVxi]);
  const T* ay = q + g.vol(0, face, g.slot[kVeta]);
  const T* ar = q + g.vol(0, face, g.slot[kVr]);
  const long long o = g.at(k, j, i);
  auto ddx = [&](const T* f) {
    double s = 0.0;
    for (int m = 1; m <= 3; ++m) s += Coef<double>::drp(m) * ((double)f[o + m] - (double)f[o - m]);
    return s * inv_dxi;
  };
  auto ddy = [&](const T* f) {
    double s = 0.0;
    for (int m = 1; m <= 3; ++m) s += Coef<double>::drp(m) * ((double)f[o + m * g.pitch] - (double)f[o - m * g.pitch]);
    return s * inv_dxi;
  };
  auto ddr = [&](const T* f) {           // DDR with the one-sided rows at both ends
    const double facr = (double)rad[rFacR * nr + k];
    const long long col = g.at(0, j, i);
    if (k >= 3 && k <= nr - 4) {
      double s = 0.0;
      for (int m = 1; m <= 3; ++m)
        s += Coef<double>::drp(m) * ((double)f[col + (k + m) * g.plane] - (double)f[col + (k - m) * g.plane]);
      return facr * s;
    }
    const bool lo = k < 3;
    const int brow = lo ? k : nr - 1 - k, ks = lo ? 0 : nr - 7;
    double s = 0.0;
    for (int p = 0; p < 7; ++p) s += Coef<double>::bdy(brow, lo ? p : 6 - p) * (double)f[col + (long long)(ks + p) * g.plane];
    return lo ? facr * s : -facr * s;
  };
  const double X = tanx[i], Y = tanx[j];
  const double C = sqrt(1.0 + X * X), D = sqrt(1.0 + Y * Y), sd = sqrt(1.0 + X * X + Y * Y);
  const double XY = X * Y, CD = C * D, rk = gr[k];
  const double axv = (double)ax[o], ayv = (double)ay[o];
  const double d_r_xi = ddx(ar), d_r_eta = ddy(ar);
  const double d_xi_xi = ddx(ax), d_eta_eta = ddy(ay), d_eta_xi = ddx(ay), d_xi_eta = ddy(ax);
  const double d_xi_r = ddr(ax), d_eta_r = ddr(ay);
  const double cx = XY / sd * d_xi_r - CD / sd * d_eta_r + (1.0 / rk) * (XY / sd * axv - CD / sd * ayv + sd / D * d_r_eta);
  const double ce = CD / sd * d_xi_r - XY / sd * d_eta_r + (1.0 / rk) * (CD / sd * axv - XY / sd * ayv - sd / C * d_r_xi);
  const double crr = (sd / rk) * (XY / CD * (d_eta_eta / D - d_xi_xi / C) - d_xi_eta / D + d_eta_xi / C);
  out[g.vol(0, face, g.slot[kVxi]) + o] = (T)cx;
  out[g.vol(0, face, g.slot[kVeta]) + o] = (T)ce;
  out[g.vol(0, face, g.slot[kVr]) + o] = (T)crr;
}

template <typename T>
static int enqueue_curl(solar_ctx* c) {
  const Geom& g = c->g;
  curl_edge_kernel<T><<<dim3((unsigned)((g.n + 127) / 128), 72, (unsigned)g.nr), 128, 0, c->stream>>>(
      (T*)c->B, (const T*)c->dt.ew, (const T*)c->dt.egc, c->dt.s0t, g);
  const long long n6 = 6LL * g.n * g.n * g.nr;
  curl_kernel<T><<<(unsigned)((n6 + 255) / 256), 256, 0, c->stream>>>((const T*)c->B, (T*)c->W, c->dt.tanx, c->dt.gr,
                                                                      (const T*)c->dt.rad, g, 1.0 / c->ht.dxi);
  CK(cudaGetLastError());
  return SOLAR_OK;
}

}  // namespace solar

extern "C" {

int solar_gpu_curl(solar_ctx* c, const double* a_xi, const double* a_eta, const double* a_r, double* curl_xi,
                   double* curl_eta, double* curl_r) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!a_xi || !a_eta || !a_r || !curl_xi || !curl_eta || !curl_r) return fail(SOLAR_ERR_ARG, "null array");
  if (c->g.nface != 6) return fail(SOLAR_ERR_ARG, "the curl needs a context owning all six zones");
  if (!c->dt.egc) {
    rc = c->fp32 ? upload<float>(&c->dt.egc, c->ht.egc) : upload<double>(&c->dt.egc, c->ht.egc);
    if (rc) return rc;
  }
  const int fx = kVxi, fy = kVeta, fr = kVr;
  if ((rc = upload_fields(c, c->B, 0, a_xi, 1, &fx, 1))) return rc;
  if ((rc = upload_fields(c, c->B, 0, a_eta, 1, &fy, 1))) return rc;
  if ((rc = upload_fields(c, c->B, 0, a_r, 1, &fr, 1))) return rc;
  rc = c->fp32 ? enqueue_curl<float>(c) : enqueue_curl<double>(c);
  if (rc) return rc;
  if ((rc = download_fields(c, c->W, 0, curl_xi, 1, &fx, 1))) return rc;
  if ((rc = download_fields(c, c->W, 0, curl_eta, 1, &fy, 1))) return rc;
  return download_fields(c, c->W, 0, curl_r, 1, &fr, 1);
}

}  // extern "C"
