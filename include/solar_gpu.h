/*
 * solar_gpu.h -- C-ABI of the B200 (sm_100a) time-stepping engine for the cubed-sphere
 * linear-acoustics solver ankitvb/solar.
 *
 * The reference is Fortran 90 + MPI.  Its time-stepping path is a link-time plug-in
 * surface (makefile:14-18): external subroutines RK4 (timestep.f90:41), COMPUTE_RHS
 * (compute_rhs_acoustic.f90:1), BC_RHS (bc_acoustic_wave.f90:1), SPONGE (sponge.f90:1)
 * and the module procedure FILTER_EXP (filter.f90:9), all working on the state
 * q(mx,my,mr,5) of COMMON /RKWORK/ (cube.f90:18-20).  This header is the C side of that
 * surface for a host that drives all six cubed-sphere faces from one process: every
 * entry point takes plain pointers and sizes, returns an int status and never aborts.
 *
 * Array layout of every host array below (FP64, "six-zone Fortran order"): the six
 * per-zone Fortran arrays concatenated in zone order 1..6,
 *    field arrays   f[zone][k][j][i]          = f(mx,my,mr) of each zone, i fastest
 *    state arrays   q[zone][m][k][j][i]       = q(mx,my,mr,5) of each zone,
 *                                               m = rho, v_xi, v_eta, v_r, p
 * with mx = my = nx and mr = nr (the reference's px = py = pr = 1 case).  A Fortran
 * host with one zone per rank passes its q(:,:,:,:) directly for one zone slot.
 *
 * Threading: a context belongs to one host thread and one CUDA device; calls are
 * stream-ordered on the context's own stream and complete before they return.
 */
#ifndef SOLAR_GPU_H
#define SOLAR_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define SOLAR_GPU_ABI_VERSION 1

/* Status codes.  SOLAR_ERR_* are negative; solar_gpu_last_error() has the detail. */
#define SOLAR_OK 0
#define SOLAR_ERR_ARG (-1)      /* bad argument or unsupported size                  */
#define SOLAR_ERR_CUDA (-2)     /* a CUDA runtime call failed                        */
#define SOLAR_ERR_NAN (-3)      /* the NaN/Inf watchdog tripped                      */
#define SOLAR_ERR_TIMEOUT (-4)  /* a bounded device wait gave up                     */
#define SOLAR_ERR_STATE (-5)    /* context not initialised / wrong call order        */
#define SOLAR_ERR_NOMEM (-6)    /* device or pinned host allocation failed           */

#define SOLAR_FP64 0            /* state, stencils and accumulation in double        */
#define SOLAR_FP32 1            /* state and stencils in float; metric, interpolation
                                   weights and diagnostics computed once in double   */

typedef struct solar_ctx solar_ctx;

/* Run configuration.  Everything the reference fixes at compile time in 'header'
 * (header:4-10) or hard-codes in the plug-ins becomes a field here; the defaults from
 * solar_desc_defaults() equal the reference's values. */
typedef struct solar_desc {
  int nx;          /* points per face edge, nx = ny (header:4); multiple of 16, >= 16      */
  int nr;          /* radial points (header:4); >= 16                                      */
  int precision;   /* SOLAR_FP64 | SOLAR_FP32                                               */
  int nfields;     /* 5: the reference's (rho, v, p).  4: rho dropped -- only valid when
                      g0 == 0, where rho is write-only (compute_rhs_acoustic.f90:83, 146)  */
  int nruns;       /* independent runs held side by side (batched sources); >= 1          */
  int device;      /* CUDA device ordinal                                                  */
  double dt;       /* deltat; the reference overrides its CFL estimate (timestep.f90:35),
                      so the host sets it                                                  */
  const double* model;   /* nr x 8 'solar_model' rows, row-major (r/R, c, rho, p, T, g,
                            Gamma, unused), normalised here as SOLAR_DATA does
                            (ic_acoustic_wave.f90:73-108)                                   */
  const double* c2_3d;   /* optional six-zone field of c^2 replacing the radial c^2 (a 3-D
                            sound-speed perturbation); NULL = radial background            */
  double sponge_amp;     /* a_sponge = 0.1   (sponge.f90:20)                               */
  double sponge_exp;     /* s_exp = 3        (sponge.f90:21)                               */
  int sponge_len;        /* k_sponge_length = 30 (sponge.f90:27)                           */
  int sponge_lower;      /* keep the inner-end branch (sponge.f90:42-43); default 1        */
  int sponge_upper;      /* keep the outer-end branch (sponge.f90:40-41); default 1        */
  int fix_reversed_rotation; /* 0 (default) = reference arithmetic.  1 = evaluate the
                            receiver-frame rotation of the eight reversed vector strips
                            (transform.f90:184-274) at the receiver's mirrored edge index  */
  int tile_x, tile_y, kchunk; /* stage-kernel tile (16x16, 32x8, 32x16 or 64x8) and radial
                                planes per CTA; 0 = default: 64x8 when nx is a multiple of
                                64, else 32x16 (float) / 32x8 (double), 16x16 when nx is
                                not a multiple of 32; nr/3 (float) or nr/6 (double) planes,
                                clamped to 16..64 (finer when that would not fill one wave
                                of two CTAs per SM).  solar_b200/autotune.py measures the
                                best for a workload.                                         */
} solar_desc;

/* Fill *d with the reference's defaults (sizes 0, FP64, 5 fields, 1 run, device 0,
 * sponge 0.1 / 3 / 30 at both ends). */
void solar_desc_defaults(solar_desc* d);

/* Setup sequence of cube.f90:35-51 (SOLAR_DATA, SETUP_COORDINATES_METRICS_ALL,
 * SETUP_LAGRANGE_INTERPOLANT): builds the FP64 metric, background, interpolation and
 * edge-rotation tables on the host, uploads them, and allocates the device state.  The
 * state starts at zero (GENERATE_IC, ic_acoustic_wave.f90:4-29). */
int solar_gpu_init(const solar_desc* d, solar_ctx** out);

/* Release every device and host resource of the context. */
int solar_gpu_finalize(solar_ctx* c);

/* COMMON /RKWORK/ q (cube.f90:18-20): copy one run's state in / out, six-zone Fortran
 * order, 6*5*nr*nx*nx doubles.  With nfields = 4 the rho slot reads back as 0. */
int solar_gpu_set_state(solar_ctx* c, int run, const double* q);
int solar_gpu_get_state(solar_ctx* c, int run, double* q);

/* IC plug-in (GENERATE_IC slot, makefile:16): p += amp exp(-|x-x0|^2 / (2 width^2)) at
 * the grid points x = r (unit vector of the zone's cube point). */
int solar_gpu_add_gaussian(solar_ctx* c, int run, double x0, double y0, double z0,
                           double width, double amp);

/* RK4 (timestep.f90:41-86): nsteps calls of the reference's RK4 -- five 2N-storage
 * stages of COMPUTE_RHS + BC_RHS + SPONGE + update, then FILTER_EXP -- on every run. */
int solar_gpu_rk4(solar_ctx* c, int nsteps);

/* Batched RK4: run r advances nsteps_per_run[r] steps (uneven counts), all live runs in the
 * same launches.  Runs are ordered by step count; each stretch of steps with the same number
 * of live runs replays one captured CUDA graph whose grids cover only those runs (graphs are
 * kept per live-run count). */
int solar_gpu_rk4_runs(solar_ctx* c, const int* nsteps_per_run);

/* solar_gpu_rk4_runs, plus the device time of the whole batch (CUDA events on the
 * context's stream) in *ms. */
int solar_gpu_time_rk4_runs(solar_ctx* c, const int* nsteps_per_run, double* ms);

/* Operator-level drop-ins (host arrays in, host arrays out; use run 0's buffers):
 *   COMPUTE_RHS (compute_rhs_acoustic.f90:1-159; source term as set) q -> rhs
 *   BC_RHS      (bc_acoustic_wave.f90:1-36)                          rhs in place
 *   SPONGE      (sponge.f90:1-58)                                    q, rhs in place
 *   FILTER_EXP  (filter.f90:9-48)                                    q -> qf
 *   COMPUTE_GRADIENT  (grad.f90:13-59)     field p -> (grad_xi, grad_eta, grad_r)
 *   COMPUTE_DIVERGENCE (grad.f90:62-136)   fields (v_xi, v_eta, v_r) -> div        */
int solar_gpu_compute_rhs(solar_ctx* c, const double* q, double* rhs);
int solar_gpu_bc_rhs(solar_ctx* c, double* rhs);
int solar_gpu_sponge(solar_ctx* c, const double* q, double* rhs);
int solar_gpu_filter_exp(solar_ctx* c, const double* q, double* qf);
int solar_gpu_gradient(solar_ctx* c, const double* p, double* grad_xi, double* grad_eta,
                       double* grad_r);
int solar_gpu_divergence(solar_ctx* c, const double* v_xi, const double* v_eta,
                         const double* v_r, double* div);

/* COMPUTE_CURL (grad.f90:140-255) with its halo transform TRANSFORM_VECTOR_BETWEEN_MESHES_CURL
 * (transform.f90:279-498): (a_xi, a_eta, a_r) -> (curl_xi, curl_eta, curl_r), six-zone fields.
 * Not used by the acoustics; the reference's defect on the eight reversed strips applies
 * here too, and fix_reversed_rotation removes it. */
int solar_gpu_curl(solar_ctx* c, const double* a_xi, const double* a_eta, const double* a_r, double* curl_xi,
                   double* curl_eta, double* curl_r);

/* norm (auxiliary.f90:100-125) of field m (1..5) of one run, in double:
 * (sum(f^2) / (nx*ny*nr) * 6)^0.5 over the six zones, the reference's formula. */
int solar_gpu_norm(solar_ctx* c, int run, int field, double* out);

/* The same norm of a six-zone FP64 field f[zone][k][j][i] that already lives in device
 * memory, for callers that cannot allocate (a host whose device memory is budgeted by
 * another runtime, or a per-step diagnostic hook that must not trigger the device-wide
 * synchronisation of cudaMalloc/cudaFree).  No counterpart in the reference: it has no
 * device.  Allocates nothing: its scratch is a fixed 96 KiB device array inside the
 * library, so nr <= 2048 and nx * nx <= INT_MAX (larger grids return SOLAR_ERR_ARG before
 * any launch).  d_out is one device double; the call only enqueues work on `stream` (a
 * cudaStream_t, NULL = legacy default stream).  The first call in each CUDA context
 * resolves the scratch address (again after a cudaDeviceReset) and should come before any
 * stream capture.  Calls whose kernels overlap on the same device race on the shared
 * scratch. */
int solar_gpu_norm_noalloc(const double* d_field, int nx, int nr, double* d_out, void* stream);

/* cube.f90:71-79 loop body without the host waits: nsteps calls of RK4 (as solar_gpu_rk4)
 * and after each the norm (auxiliary.f90:100-125, as solar_gpu_norm) of field m (1..5) of
 * one run.  norms[s] = the norm after step s+1.  The per-step sums stay on the device and
 * are read back once at the end, so the host does not wait on the GPU between steps. */
int solar_gpu_rk4_norms(solar_ctx* c, int run, int field, int nsteps, double* norms);

/* NaN/Inf watchdog.  No counterpart in the reference, which only prints norm(v_r) after
 * each step (cube.f90:77).  With every > 0, solar_gpu_rk4, solar_gpu_rk4_runs,
 * solar_gpu_rk4_norms, solar_gpu_time_rk4 and solar_gpu_step_phase scan the state buffer
 * for non-finite values after every `every`-th step of the context (one read of the state,
 * enqueued without a host wait); the call then returns SOLAR_ERR_NAN and
 * solar_gpu_last_error names the first step (counted over the context's life) at which a
 * non-finite value was seen.  every = 0 (the default) switches it off. */
int solar_gpu_set_watchdog(solar_ctx* c, int every);

/* Failure-detection test hook.  No counterpart in the reference.  Every wait of a
 * streaming kernel on its shared-memory load ring is bounded (2^22 polls of
 * mbarrier.try_wait, about a second or more); a kernel whose wait gives up stops issuing
 * loads, waits (bounded) for the loads it issued, exits, and the call returns
 * SOLAR_ERR_TIMEOUT.  With kernels != 0 the named kernels issue no loads at all and give up
 * after `polls` polls (1 .. 2^22), so their first wait runs out with nothing in flight;
 * kernels = 0 restores normal operation.  Captured step graphs are rebuilt. */
#define SOLAR_KERNEL_EDGE 1
#define SOLAR_KERNEL_STAGE 2
#define SOLAR_KERNEL_FILTER 4
#define SOLAR_KERNEL_ADJ_STAGE 8
int solar_gpu_inject_wait_timeout(solar_ctx* c, int kernels, int polls);

/* FP64 diagnostics of one run: out[0] = acoustic energy
 * 1/2 sum (rho0 |v|^2 + p^2 / (rho0 c^2)) dV, out[1] = sum rho dV, out[2] = max |p|,
 * out[3] = 1 if any value is NaN/Inf.  dV is the cubed-sphere volume element
 * r^2 (1+X^2)(1+Y^2) / delta^(3/2) dxi deta dr. */
int solar_gpu_diag(solar_ctx* c, int run, double* out4);

/* Timed helpers for benchmarks: run nsteps of solar_gpu_rk4 with CUDA events on the
 * context's stream.  out[0] = total ms; with per_kernel != 0 the steps are launched
 * without the CUDA graph and out[1..3] = mean ms per launch of the stage, filter and
 * edge kernels, out[4..6] = launches of each kind. */
int solar_gpu_time_rk4(solar_ctx* c, int nsteps, int per_kernel, double* out7);

/* Block until the context's stream is idle. */
int solar_gpu_synchronize(solar_ctx* c);

/* ---- Source term of the v_r equation (nruns == 1) ------------------------------------
 * SOLAR_FORCING_ANALYTIC: compute_rhs_acoustic.f90:92-104, S = mag(t) exp(-((theta-pi/2)/
 *   (20 dxi))^2 - (phi/(20 dxi))^2 - ((r-r_c)/(20 dchi))^2) with mag(t) = exp(-(tau-650)^2/
 *   (2*200^2)) cos(4 pi (tau-650)/700), tau = t rsun/c(row 1).  r_c = r of plane k_center
 *   (0-based; the reference hard-codes gr(200), i.e. k_center = 199).
 * SOLAR_FORCING_SAMPLES: the sampled source S_t(x,y,n) (READ_FORCING_FUNC, output.f90:271-
 *   307) interpolated in time by LAGRANGE_INTERP (interpolation.f90:385-451) and added at
 *   the plane e_rad (r nearest 1 - 100 km/R_sun), as the commented block of
 *   compute_rhs_acoustic.f90:107-116 does; nstep is the run's step count (cube.f90:71),
 *   which LAGRANGE_INTERP uses to drop its last two nodes.
 * Every stage of one RK4 call uses the call's time; RK4 advances time by dt and the step
 * counter by one (timestep.f90:82).  The clock starts at time 0, step 0. */
#define SOLAR_FORCING_OFF 0
#define SOLAR_FORCING_ANALYTIC 1
#define SOLAR_FORCING_SAMPLES 2
int solar_gpu_set_forcing(solar_ctx* c, int kind, int k_center, int nstep);
/* Samples of one zone in the file order of READ_FORCING_FUNC: f[(i*ny + j)*nt + n]. */
int solar_gpu_set_forcing_samples(solar_ctx* c, int zone, const double* f, int nt);
/* READ_FORCING_FUNC (output.f90:271-307): the six files dir/forcing/forcing_cubesph.<z+1>,
 * each one unformatted record of nx*nx*nt float64 values, into the sampled source. */
int solar_gpu_load_forcing(solar_ctx* c, const char* dir, int nt);
int solar_gpu_set_clock(solar_ctx* c, double time, int step);
int solar_gpu_get_clock(solar_ctx* c, double* time, int* step);

/* ---- Zones split across processes (one GPU per process, nruns == 1) ---------------
 * The reference runs one MPI rank per zone block and exchanges interpolated halo strips
 * inside every derivative (derivative.f90:8-323).  Here a context can own a contiguous
 * range of zones: the step kernels then run on those zones only.  Every ghost value of an
 * owned zone is interpolated from the three lines next to one edge of a neighbouring zone
 * (the route table); where that zone belongs to another process, the host moves those
 * lines between the phases of a step: pack on the owner, transfer (e.g. NCCL send/recv on
 * the context's stream), unpack on the receiver, then run the phase.
 *
 * Owned zones zone0 .. zone0+nzones-1 (0-based); the default is all six.  Diagnostics
 * (solar_gpu_norm, solar_gpu_diag) then cover the owned zones only. */
int solar_gpu_set_owned_zones(solar_ctx* c, int zone0, int nzones);

/* routes[(z*4+e)*3 + {0,1,2}] = (source zone, source edge, reversed) of the ghost frame of
 * zone z (0-based) at edge e (0 S, 1 N, 2 W, 3 E): derivative.f90's halo routing. */
int solar_gpu_edge_routes(int* routes);

/* One phase of an RK4 call, enqueued on the context's stream (no wait): phases 0..4 are
 * the five stages (edge exchange of p, v_xi, v_eta + fused stage kernel), phase 5 is
 * FILTER_EXP (edge exchange of every field + filter).  Phases 0..5 in order = one
 * solar_gpu_rk4(c, 1).  Phases 6 and 7 are the two halves of phase 5 (edge exchange; filter),
 * between which a process owning a radial slab receives its neighbours' boundary planes. */
int solar_gpu_step_phase(solar_ctx* c, int phase);

/* Stage phase p (0..4) in two parts, so that the edge-line exchange of the phase can be in
 * transit while part 0 runs; the reference overlaps its halo messages with the interior
 * the same way (derivative.f90:135-148).  Part 0: the stage kernel on the interior tiles,
 * which read no ghost frame and no line of another zone.  Part 1: the edge kernel, then the
 * stage kernel on the tiles along the face edges.  Issue part 0 before part 1, with the
 * phase's radial boundary planes already in place; unpack the received lines between the
 * two.  Parts 0 and 1 together equal solar_gpu_step_phase(c, p) bit for bit.  A face of
 * fewer than 3 x 3 stage tiles has no interior: part 0 then launches nothing. */
int solar_gpu_step_phase_part(solar_ctx* c, int phase, int part);

/* ---- Radial slabs (the reference's pr decomposition, header:6; nruns == 1) -------------
 * The step kernels compute planes k0 .. k1-1 only (k1 - k0 >= 5; default 0 .. nr-1).  The
 * radial stencils near a slab boundary read the neighbouring slab's planes, which the host
 * moves between the phases of a step (derivative.f90:605-758 exchanges 3 planes for DDR,
 * filter.f90:633-781 5 planes for FILTER_R): before stage phase p (0..4) the 3 planes of p and
 * v_r next to each boundary, before the filter (between phases 6 and 7) the 5 planes of every
 * stored field, frames included.  Zones and slabs combine: a process owns a zone range and a
 * plane range; the edge lines of solar_gpu_pack_lines then cover the owned planes only. */
int solar_gpu_set_owned_planes(solar_ctx* c, int k0, int k1);

/* Values (of the context's precision) one phase sends to one radial neighbour: owned zones x
 * fields (2 before a stage, nfields before the filter) x planes (3 / 5) x padded plane. */
long long solar_gpu_planes_size(solar_ctx* c, int phase);

/* side 0: the neighbour below (sends planes k0 .. k0+H-1, receives k0-H .. k0-1);
 * side 1: the neighbour above (sends k1-H .. k1-1, receives k1 .. k1+H-1).  phase 0..5 names
 * the exchange (5 = the filter's).  Enqueued on the context's stream. */
int solar_gpu_pack_planes(solar_ctx* c, int phase, int side, void* d_buf);
int solar_gpu_unpack_planes(solar_ctx* c, int phase, int side, const void* d_buf);

/* Values (of the context's precision) in the packed lines of one (zone, edge) pair in
 * phase `phase`: 3 * nx * nr * (3 fields in phases 0..4, every stored field in phase 5). */
long long solar_gpu_lines_size(solar_ctx* c, int phase);

/* Copy the source lines of `count` (zone, edge) pairs (zone_edge[2q], zone_edge[2q+1]) of
 * the buffer that phase `phase` reads into / out of the device buffer d_buf
 * (count * solar_gpu_lines_size values).  Enqueued on the context's stream. */
int solar_gpu_pack_lines(solar_ctx* c, int phase, const int* zone_edge, int count, void* d_buf);
int solar_gpu_unpack_lines(solar_ctx* c, int phase, const int* zone_edge, int count, const void* d_buf);

/* The context's CUDA stream (a cudaStream_t), to order the caller's transfers with it. */
void* solar_gpu_stream(solar_ctx* c);

/* Raw partial sums over the owned zones of run `run`, for a cross-process reduction:
 * out5 = (sum of field^2 (field 1..5; 0 = none), energy, mass, max |p|, non-finite count). */
int solar_gpu_reduce_owned(solar_ctx* c, int run, int field, double* out5);

/* ---- The reference's output files (output.f90), for the zones of run `run` ------------
 * Paths are relative to `dir` (the reference writes into its working directory); missing
 * directories are created.  Zone z (0-based) is the reference's rank z and zone z+1 of the
 * px = py = pr = 1 layout.  NNN is the three-digit cue (dirs.c:20).
 *   restart  WRITE_RESTART (output.f90:86-190): dir/Restart/restart.NNN.<z+1>, a 28-byte
 *            header (int32 nx, ny, nr, 5; float64 time; int32 step) then q(nx,ny,nr,5)
 *            float64 in Fortran order.  The reference has no reader; solar_gpu_read_restart
 *            loads the same files into the state (header checked against the context).
 *   visual   WRITE_VISUAL (output.f90:192-240): dir/Visual/NNN/vis_<z>, one Fortran
 *            unformatted record (4-byte length markers) of q(:,:,o_rad,1:5).
 *   grid     WRITE_GRID (output.f90:242-267): dir/Visual/grid/grid_<z>, FORMAT(1x,7i5).
 *   trace    WRITE_RADIAL_TRACE (output.f90:309-343): appends ((q(1,1,k,l),k=1,nr),l=1,5)
 *            to dir/trace_<z+1> with FORMAT(1x,5(ES13.5)). */
int solar_gpu_write_restart(solar_ctx* c, int run, const char* dir, int cue, double time, int step);
int solar_gpu_read_restart(solar_ctx* c, int run, const char* dir, int cue, double* time, int* step);
int solar_gpu_write_visual(solar_ctx* c, int run, const char* dir, int cue);
int solar_gpu_write_grid(solar_ctx* c, const char* dir);
int solar_gpu_write_radial_trace(solar_ctx* c, int run, const char* dir);

/* o_rad of SOLAR_DATA (ic_acoustic_wave.f90:124-132), 0-based: the plane WRITE_VISUAL dumps. */
int solar_gpu_output_plane(solar_ctx* c, int* k);

/* The same formats for one zone from host arrays (no device needed). */
int solar_io_cue_name(int cue, char* buf, int len);
int solar_io_format_es(double v, int w, int d, char* out);          /* Fortran ESw.d, out: w+1 chars */
int solar_io_write_restart(const char* path, const double* q, int nx, int ny, int nr, double time, int step);
int solar_io_read_restart(const char* path, double* q, int nx, int ny, int nr, double* time, int* step);
int solar_io_write_visual(const char* path, const double* plane5, int nx, int ny);
int solar_io_write_grid(const char* path, const int* seven);
int solar_io_append_trace(const char* path, const double* values, int count);
int solar_io_read_forcing(const char* path, int nx, int ny, int nt, double* f);

/* ---- Discrete adjoint (run 0 of a context with nruns == 1) -------------------------
 * No counterpart in the reference, which has no adjoint.  These are the exact transposes
 * of the discrete forward operators above: COMPUTE_RHS + BC_RHS + SPONGE, FILTER_EXP
 * (with the halo interpolation and vector rotation of the edge exchange) and the 2N-RK
 * step of timestep.f90:61-82 run backwards stage by stage.  Host arrays use the
 * six-zone Fortran order of the header comment.
 *
 * Receivers sample p with trilinear weights on one face: loc[4*r .. 4*r+3] =
 * (zone 0..5, i, j, k) as fractional 0-based grid indices (i along xi, j along eta,
 * k along the radius), each inside [0, nx-1] x [0, nx-1] x [0, nr-1]. */
int solar_gpu_set_receivers(solar_ctx* c, int nrec, const double* loc);

/* nsteps forward steps from the current state; traces[n*nrec + r] = p at receiver r
 * after step n+1.  Leaves the state at step nsteps. */
int solar_gpu_record(solar_ctx* c, int nsteps, double* traces);

/* Misfit J = 1/2 sum_{n=1..nsteps} sum_r (p_r(t_n) - data[(n-1)*nrec + r])^2 of an
 * nsteps-step run from the current state, and its gradient with respect to the sound
 * speed c at every grid point: grad_c[zone][k][j][i] = dJ/dc (0 on the two radial
 * boundary planes, where BC_RHS discards the right-hand side).  The state is
 * checkpointed every `checkpoint_every` steps; each segment is recomputed once during
 * the reverse sweep, storing the divergence of its stage inputs (memory: one state per
 * checkpoint plus 5 * checkpoint_every field volumes).  Optional outputs (may be NULL):
 * misfit, grad_c, lambda0 = dJ/dq at the initial state (state array), times_ms[3] =
 * device time of the forward sweep, the recomputation and the reverse sweep.  On
 * return the state is back at the initial condition. */
int solar_gpu_misfit_gradient(solar_ctx* c, int nsteps, int checkpoint_every, const double* data,
                              double* misfit, double* grad_c, double* lambda0, double* times_ms);

/* solar_gpu_misfit_gradient with two checkpoint levels, for grids whose single-level
 * checkpoints do not fit: states are kept every checkpoint_every steps for the whole run;
 * each of those segments is run forward once more keeping a state every inner_every steps,
 * and only those inner segments store stage divergences (memory: one state per outer and
 * per inner checkpoint plus 5 * inner_every field volumes; cost: one more forward run).
 * inner_every >= checkpoint_every is the single-level sweep. */
int solar_gpu_misfit_gradient_nested(solar_ctx* c, int nsteps, int checkpoint_every, int inner_every,
                                     const double* data, double* misfit, double* grad_c, double* lambda0,
                                     double* times_ms);

/* out = L^T mu, L(q) = SPONGE(BC_RHS(COMPUTE_RHS(q))) as a linear map of the state. */
int solar_gpu_rhs_adjoint(solar_ctx* c, const double* mu, double* out);

/* out = FILTER_EXP^T lam (halo interpolation included). */
int solar_gpu_filter_adjoint(solar_ctx* c, const double* lam, double* out);

/* lam_out = (STEP^T)^nsteps lam_in, STEP = one RK4 call (five stages + FILTER_EXP). */
int solar_gpu_rk4_adjoint(solar_ctx* c, int nsteps, const double* lam_in, double* lam_out);

/* Copy the last error message of this thread (NUL-terminated, truncated to len). */
int solar_gpu_last_error(char* buf, int len);

/* ABI version (SOLAR_GPU_ABI_VERSION). */
int solar_gpu_abi_version(void);

/* Name of CUDA device `device` (NUL-terminated, truncated to len); used to key tuned
 * launch shapes.  No counterpart in the reference (it has no device). */
int solar_gpu_device_name(int device, char* buf, int len);

#ifdef __cplusplus
}
#endif
#endif /* SOLAR_GPU_H */
