// split_host.cuh -- zones split across processes (one GPU each): owned-zone range, the
// phases of one RK4 call, and packing of the edge lines that neighbouring zones on other
// processes interpolate their ghost values from.  Included once, by solar_gpu.cu.
//
// The reference runs one MPI rank per zone block and exchanges interpolated halo strips
// inside every derivative (derivative.f90:8-323 with MPI_INTERCOMM sends/receives).  Here
// a process owns a contiguous range of zones and runs the same fused kernels on them; the
// exchange moves the raw source lines (three lines next to each edge) once per phase, and
// each receiver interpolates and rotates them with its own edge kernel.
#pragma once

namespace solar {

static int split_items_upload(solar_ctx* c, const int* zone_edge, int count) {
  if (count < 0 || count > 24 || (count && !zone_edge)) return fail(SOLAR_ERR_ARG, "need 0..24 (zone, edge) pairs");
  for (int q = 0; q < count; ++q) {
    const int z = zone_edge[2 * q], e = zone_edge[2 * q + 1];
    if (z < 0 || z > 5 || e < 0 || e > 3) return fail(SOLAR_ERR_ARG, "bad (zone, edge) pair (%d, %d)", z, e);
  }
  if (!c->split_items) {
    CK(cudaMalloc((void**)&c->split_items, 48 * sizeof(int)));
    CK(cudaMalloc((void**)&c->split_slots, 8 * sizeof(int)));
    int sl[8] = {c->g.slot[kP], c->g.slot[kVxi], c->g.slot[kVeta], 0, 1, 2, 3, 4};
    CK(cudaMemcpy(c->split_slots, sl, sizeof(sl), cudaMemcpyHostToDevice));
  }
  if (count) CK(cudaMemcpyAsync(c->split_items, zone_edge, 2 * count * sizeof(int), cudaMemcpyHostToDevice, c->stream));
  return SOLAR_OK;
}

static int phase_slots(const solar_ctx* c, int phase) { return phase == 5 ? c->g.nf : 3; }

// buffer read by phase p's edge kernel: A, B, A, B, A for the stages, B for the filter
static void* phase_buffer(solar_ctx* c, int phase) { return (phase == 5 || phase % 2) ? c->B : c->A; }

static int lines_op(solar_ctx* c, int phase, const int* zone_edge, int count, void* d_buf, int unpack) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (phase < 0 || phase > 5) return fail(SOLAR_ERR_ARG, "phase must be 0..5");
  if (c->g.nruns != 1) return fail(SOLAR_ERR_ARG, "zone splitting needs nruns == 1");
  if (count && !d_buf) return fail(SOLAR_ERR_ARG, "null device buffer");
  if ((rc = split_items_upload(c, zone_edge, count))) return rc;
  if (!count) return SOLAR_OK;
  const int ns = phase_slots(c, phase);
  const int* slots = c->split_slots + (phase == 5 ? 3 : 0);
  const long long total = 3LL * c->g.n * (c->g.k1 - c->g.k0) * ns * count;
  const unsigned blocks = (unsigned)((total + 255) / 256);
  void* q = phase_buffer(c, phase);
  if (c->fp32)
    line_pack_kernel<float><<<blocks, 256, 0, c->stream>>>((const float*)q, (float*)d_buf, c->split_items, count,
                                                           slots, ns, c->g, unpack);
  else
    line_pack_kernel<double><<<blocks, 256, 0, c->stream>>>((const double*)q, (double*)d_buf, c->split_items, count,
                                                            slots, ns, c->g, unpack);
  CK(cudaGetLastError());
  return SOLAR_OK;
}

// Phases 0..4: edge exchange + stage s; 5: edge exchange + FILTER_EXP; 6 and 7: the two
// halves of phase 5 (a process owning a radial slab receives its neighbours' boundary
// planes, frames included, between them).
template <typename T>
static int enqueue_phase(solar_ctx* c, int phase) {
  int rc;
  if (phase == 0 && (rc = force_begin(c))) return rc;
  if (phase < 5) {
    void* in = phase % 2 ? c->B : c->A;
    void* out = phase % 2 ? c->A : c->B;
    if ((rc = launch_edge<T>(c, in, 0, nullptr))) return rc;
    return launch_stage<T>(c, in, out, phase == 0 ? 1 : 0, phase, nullptr);
  }
  if (phase != 7 && (rc = launch_edge<T>(c, c->B, 1, nullptr))) return rc;
  if (phase == 6) return SOLAR_OK;
  if ((rc = launch_filter<T>(c, c->B, c->A, nullptr))) return rc;
  return force_end(c);
}

// Phases 0..4 in two parts, so that a process can overlap the edge-line exchange with
// computation.  Part 0: the stage on the interior tiles, which read no ghost frame and no
// line of another zone (phase 0 also starts the step's forcing).  Part 1: the edge kernel,
// then the stage on the ring of face-edge tiles.  Part 0 precedes part 1; the radial slab's
// boundary planes of the phase must be in place before part 0, the received edge lines
// before part 1.  The two parts write disjoint points, so together they equal the phase.
template <typename T>
static int enqueue_phase_part(solar_ctx* c, int phase, int part) {
  int rc;
  void* in = phase % 2 ? c->B : c->A;
  void* out = phase % 2 ? c->A : c->B;
  const int mode = phase == 0 ? 1 : 0;
  if (part == 0) {
    if (phase == 0 && (rc = force_begin(c))) return rc;
    return launch_stage<T>(c, in, out, mode, phase, nullptr, nullptr, kTilesInterior);
  }
  if ((rc = launch_edge<T>(c, in, 0, nullptr))) return rc;
  return launch_stage<T>(c, in, out, mode, phase, nullptr, nullptr, kTilesRing);
}

// Boundary planes exchanged between radial slabs: before stage s the three planes of p and
// v_r next to each slab boundary (the 7-point radial windows), before FILTER_EXP the five
// planes of every stored field (the 11-point radial filter; sent after the edge exchange,
// so with their frames).  Whole padded planes of the owned zones, [zone][field][plane].
static int halo_planes(int phase) { return phase == 5 ? 5 : 3; }
static int halo_fields(const solar_ctx* c, int phase, int* slots) {
  if (phase == 5) {
    for (int s = 0; s < c->g.nf; ++s) slots[s] = s;
    return c->g.nf;
  }
  slots[0] = c->g.slot[kP];
  slots[1] = c->g.slot[kVr];
  return 2;
}

static int planes_op(solar_ctx* c, int phase, int side, void* d_buf, int unpack) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (phase < 0 || phase > 5 || side < 0 || side > 1) return fail(SOLAR_ERR_ARG, "phase must be 0..5, side 0 or 1");
  if (c->g.nruns != 1) return fail(SOLAR_ERR_ARG, "radial slabs need nruns == 1");
  if (!d_buf) return fail(SOLAR_ERR_ARG, "null device buffer");
  const Geom& g = c->g;
  const int H = halo_planes(phase);
  if (side == 0 ? g.k0 < H : g.k1 + H > g.nr) return fail(SOLAR_ERR_ARG, "no radial neighbour on side %d", side);
  int slots[5];
  const int nfld = halo_fields(c, phase, slots);
  // sent: the owned planes next to the boundary; received: the planes just outside it
  const int k = unpack ? (side == 0 ? g.k0 - H : g.k1) : (side == 0 ? g.k0 : g.k1 - H);
  unsigned char* buf = static_cast<unsigned char*>(phase_buffer(c, phase));
  unsigned char* dev = static_cast<unsigned char*>(d_buf);
  const size_t block = (size_t)H * g.plane * c->esize;
  size_t off = 0;
  for (int f = g.face0; f < g.face0 + g.nface; ++f)
    for (int q = 0; q < nfld; ++q, off += block) {
      unsigned char* vol = buf + (size_t)(g.vol(0, f, slots[q]) + (long long)k * g.plane) * c->esize;
      if (unpack) CK(cudaMemcpyAsync(vol, dev + off, block, cudaMemcpyDeviceToDevice, c->stream));
      else CK(cudaMemcpyAsync(dev + off, vol, block, cudaMemcpyDeviceToDevice, c->stream));
    }
  return SOLAR_OK;
}

}  // namespace solar

extern "C" {

int solar_gpu_set_owned_zones(solar_ctx* c, int zone0, int nzones) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (zone0 < 0 || nzones < 1 || zone0 + nzones > 6) return fail(SOLAR_ERR_ARG, "owned zones must lie in 0..5");
  if (c->g.nruns != 1 && nzones != 6) return fail(SOLAR_ERR_ARG, "zone splitting needs nruns == 1");
  CK(cudaStreamSynchronize(c->stream));
  c->g.face0 = zone0;
  c->g.nface = nzones;
  // captured graphs hold the old launch shapes
  if (c->step_graph) { cudaGraphExecDestroy(c->step_graph); c->step_graph = nullptr; }
  drop_batch_graphs(c);
  return SOLAR_OK;
}

int solar_gpu_edge_routes(int* routes) {
  if (!routes) return fail(SOLAR_ERR_ARG, "null output");
  for (int z = 0; z < 6; ++z)
    for (int e = 0; e < 4; ++e) {
      routes[(z * 4 + e) * 3 + 0] = kRoutes[z][e].src_face;
      routes[(z * 4 + e) * 3 + 1] = kRoutes[z][e].src_edge;
      routes[(z * 4 + e) * 3 + 2] = kRoutes[z][e].reversed;
    }
  return SOLAR_OK;
}

int solar_gpu_step_phase(solar_ctx* c, int phase) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (phase < 0 || phase > 7) return fail(SOLAR_ERR_ARG, "phase must be 0..7");
  rc = c->fp32 ? enqueue_phase<float>(c, phase) : enqueue_phase<double>(c, phase);
  if (rc) return rc;
  CK(cudaGetLastError());
  return (phase == 5 || phase == 7) ? watch_after_step(c) : SOLAR_OK;
}

int solar_gpu_step_phase_part(solar_ctx* c, int phase, int part) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (phase < 0 || phase > 4) return fail(SOLAR_ERR_ARG, "phase parts exist for the stages 0..4 only");
  if (part < 0 || part > 1) return fail(SOLAR_ERR_ARG, "part must be 0 (interior tiles) or 1 (edge kernel, ring tiles)");
  rc = c->fp32 ? enqueue_phase_part<float>(c, phase, part) : enqueue_phase_part<double>(c, phase, part);
  if (rc) return rc;
  CK(cudaGetLastError());
  return SOLAR_OK;
}

int solar_gpu_set_owned_planes(solar_ctx* c, int k0, int k1) {
  int rc = check_ctx(c);
  if (rc) return rc;
  const int nr = c->g.nr;
  if (k0 < 0 || k1 > nr || k1 - k0 < 5) return fail(SOLAR_ERR_ARG, "owned planes [%d, %d) must lie in 0..%d and hold >= 5 planes", k0, k1, nr);
  if (c->g.nruns != 1 && (k0 != 0 || k1 != nr)) return fail(SOLAR_ERR_ARG, "radial slabs need nruns == 1");
  CK(cudaStreamSynchronize(c->stream));
  c->g.k0 = k0;
  c->g.k1 = k1;
  // captured graphs hold the old launch shapes
  if (c->step_graph) { cudaGraphExecDestroy(c->step_graph); c->step_graph = nullptr; }
  drop_batch_graphs(c);
  return SOLAR_OK;
}

long long solar_gpu_planes_size(solar_ctx* c, int phase) {
  if (!c || phase < 0 || phase > 5) return -1;
  int slots[5];
  return (long long)c->g.nface * halo_fields(c, phase, slots) * halo_planes(phase) * c->g.plane;
}

int solar_gpu_pack_planes(solar_ctx* c, int phase, int side, void* d_buf) {
  return planes_op(c, phase, side, d_buf, 0);
}

int solar_gpu_unpack_planes(solar_ctx* c, int phase, int side, const void* d_buf) {
  return planes_op(c, phase, side, const_cast<void*>(d_buf), 1);
}

long long solar_gpu_lines_size(solar_ctx* c, int phase) {
  if (!c || phase < 0 || phase > 5) return -1;
  return 3LL * c->g.n * (c->g.k1 - c->g.k0) * phase_slots(c, phase);
}

int solar_gpu_pack_lines(solar_ctx* c, int phase, const int* zone_edge, int count, void* d_buf) {
  return lines_op(c, phase, zone_edge, count, d_buf, 0);
}

int solar_gpu_unpack_lines(solar_ctx* c, int phase, const int* zone_edge, int count, const void* d_buf) {
  return lines_op(c, phase, zone_edge, count, const_cast<void*>(d_buf), 1);
}

void* solar_gpu_stream(solar_ctx* c) { return c ? (void*)c->stream : nullptr; }

int solar_gpu_reduce_owned(solar_ctx* c, int run, int field, double* out5) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!out5 || field < 0 || field > 5 || run < 0 || run >= c->g.nruns) return fail(SOLAR_ERR_ARG, "bad field/run");
  return reduce(c, run, field - 1, out5);
}

}  // extern "C"
